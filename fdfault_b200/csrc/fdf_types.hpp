// Shared host/device descriptors for the fdfault B200 time-stepping path.
//
// Field storage on the device (both precisions): structure of arrays over the
// whole domain, component-major, node order (i, j, k) with k fastest as in
// the reference's fields class (src/fields.cpp:87-98), except that the
// innermost stored dimension is padded to a multiple of FDF_PITCH_ALIGN
// elements so rows start on 32-byte boundaries (coalesced loads, TMA-legal
// strides).  Element (c, i, j, k) lives at c*cstride + i*s0 + j*s1 + k*s2;
// in 2D the innermost dimension is j and s2 = 0.
#pragma once

#include <cstdint>

#define FDF_MAX_BLOCKS 16
#define FDF_MAX_IFACES 16
#define FDF_PITCH_ALIGN 8

namespace fdf {

struct Layout {
    int ndim, mode;
    int nx[3];        // global node counts
    long long s0, s1, s2;
    long long cstride;  // elements per component
    int nfields;      // components carried by df (5 mode II, 3 mode III, 9 3D; 6 mode II plastic)
    int nfieldsp;     // plastic-only components (lambda, gammap [, 6 plastic strains])
    int nv, ns;       // velocity / stress component counts
    int sidx[6];      // s0 index of each stress component (fields.cpp:112-142)
};

// per-block parameters used by the volume kernels
struct BlockDev {
    int lo[3], n[3];      // first global node and node count per direction
    // x planes this process updates, block-local [xb, xe): the whole block
    // (0, n[0]) unless the domain is split into x slabs across processes;
    // planes outside it are read (ghost planes) but not written
    int xb, xe;
    double dx[3];         // computational grid spacing 1/(n-1) (block.cpp:772-774)
    double rho, lam, g;   // material
    double cp, cs, zp, zs, gamma;
    double mu, coh, beta, eta;   // Drucker-Prager parameters
    double coef[3][4];    // per direction: dt/rho/dx, dt(2G+lam)/dx, dt G/dx, dt lam/dx in reference order
    double nu;            // lam/(2(lam+G)) for the mode II plastic szz rate
    int bactive[6];       // outer face with SAT condition
    int defer[6];         // face is on an interface: update finalised by the interface kernel
    double r[6], alpha[6], theta[6];
    const double* fnx[6][3];  // unit normals on the face, [n_a][n_b]
    const double* fdl[6];     // |grad xi|/(h0 dxi) on the face
    int fn1[6];               // second extent of the face arrays
    // heterogeneous material (fields.cpp:582-711): rho, lambda, G per node at
    // mat[c * matstride + node] (the whole grid, shared by all blocks; matstride
    // is the layout's cstride), or null
    const double* mat;
    long long matstride;
    // which nodes the plastic return map visits and with which bulk modulus.
    // block::calc_plastic (block.cpp:442-589) declares `double k` and then an
    // `int k` z-loop index, so its k = lambda + 2/3 G lands in the loop index:
    // ptrunc 1 passes the modulus truncated to an integer; pvisit 0 every node,
    // 1 only the block's first z node of each column, 2 the nodes pmask marks
    // (the reference's z loop resumes at trunc(K) + 1)
    int ptrunc, pvisit;
    const unsigned char* pmask;
};

struct PertDev {
    int shaped;      // 0: constant shape (xy == 1), 1: xy array
    double t0;
    double val[9];
    const double* xy;   // spatial shape per fault node
};

// learned STZ initial guess: BF16 weights (stored as raw 16-bit words) and FP32 biases
struct MlpDev {
    const unsigned short* w1;   // [64][16]
    const unsigned short* w2;   // [64][64]
    const unsigned short* w3;   // [8][64]
    const float *b1, *b2, *b3;
};

// STZ Newton counters and solver-generated training samples (both optional)
struct StzAux {
    int learned;                       // 1: start Newton from the network's guess
    // start of the plain solve when not learned: 0 bracket midpoint with the
    // reference's derivative; 2 warm start (this node's previous converged mu,
    // mu_prev) with the reference's derivative; 3 bracket midpoint with the
    // exact derivative of the slip-rate law
    int start;
    double* mu_prev;                   // per fault node, < 0 where none yet (start 2)
    MlpDev mlp;
    unsigned long long* stats;         // [0] Newton solves, [1] iterations, [2] starts from the midpoint
    float* samples;                    // [cap][8]: 6 inputs, target logit(s)/20, converged mu
    unsigned long long* nsamples;
    unsigned long long cap;
};

struct IfaceDev {
    int kind;        // 0 locked, 1 frictionless, 2 slipweak, 3 stz
    int direction;
    int b1, b2;
    int n0, n1;
    int mlb[3];      // first node of the minus-side face (global indices)
    double cp1, cs1, zp1, zs1, cp2, cs2, zp2, zs2, gamma1, gamma2;
    const double *nx[3], *dl1, *dl2;
    double *u, *du, *v, *s, *sn, *ux, *dux, *vx, *sx, *state, *dstate, *dstatedt, *tfront;
    int nloads;
    const PertDev* loads;
    int load_file;
    const double *s1, *s2, *s3;
    int nperts;
    const PertDev* perts;
    int param_file;
    const double* par[9];
    const unsigned char* fin1;   // 1 where this interface finalises the minus-side node
    const unsigned char* fin2;
    StzAux stz;
};

// per-stage scalars
struct StageArgs {
    double dt, A, B, t;      // t = step time + C[stage]*dt
    int last;                // last stage of the step
    int plastic;             // material is plastic (last stage runs the return map)
    int roundtrip;           // exact path: replay the reference's absolute-stress output round trip
    int abs_out;             // write absolute stresses of this step to the staging buffer
    double tfront;           // time recorded by the front tracker after this step
    int front_on;
    double front_value;
    // graph replay: when set, t and tfront come from this device step counter
    // (t = step*dt + cst*dt, tfront = (step+1)*dt, the host's expressions)
    const int* step_dev;
    double cst;
    // polls of a bounded mbarrier wait in the TMA-staged kernels before they
    // give up with FDF_ERR_TIMEOUT (<= 0: the built-in limit)
    long long wait_limit;
};

enum Status : int {
    FDF_OK = 0,
    FDF_ERR_NEWTON = 1,       // Newton iteration failed (utilities.cpp:173-176)
    FDF_ERR_ZERO_DERIV = 2,   // zero derivative in Newton (utilities.cpp:134-137)
    FDF_ERR_MELT = 4,         // STZ slip rate above v1 (stz.cpp:341-344)
    FDF_ERR_NONFINITE = 8,    // NaN or Inf produced
    FDF_ERR_JACOBIAN = 16,    // non-positive Jacobian (block.cpp:1002)
    FDF_ERR_TIMEOUT = 32,     // a bounded wait for staged data ran out (kernel returned early)
};

}  // namespace fdf
