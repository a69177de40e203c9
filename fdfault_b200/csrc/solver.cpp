// Host orchestration of one fdfault problem on one GPU (see solver.hpp).
// Compiled with -ffp-contract=off: every host-side FP64 value that enters the
// device arithmetic (surfaces, grid spacing, stencil scale factors, material
// speeds, perturbation shapes, the time step) is formed in the reference's
// operation order.
#include "solver.hpp"

#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <fstream>
#include <stdexcept>
#include <unordered_map>

#include "energy.hpp"
#include "noalloc.hpp"
#include "output.hpp"

namespace fdf {

void cuda_check(cudaError_t e, const char* what) {
    if (e != cudaSuccess) throw std::runtime_error(std::string(what) + ": " + cudaGetErrorString(e));
}

namespace {

double sbp_h0(int order) { return order == 2 ? 0.5 : (order == 3 ? 17. / 48. : 13649. / 43200.); }

std::vector<double> read_doubles(const std::string& path, size_t n, size_t offset) {
    std::vector<double> v(n);
    std::ifstream in(path, std::ios::binary);
    if (!in) throw std::runtime_error("cannot open " + path);
    in.seekg((std::streamoff)(offset * sizeof(double)));
    if (!in.read(reinterpret_cast<char*>(v.data()), (std::streamsize)(n * sizeof(double))))
        throw std::runtime_error("cannot read " + std::to_string(n) + " values from " + path);
    return v;
}

int other_dims(int d, int& o0, int& o1) {
    o0 = (d == 0) ? 1 : 0;
    o1 = (d == 2) ? 1 : 2;
    return 0;
}

// pert::xyfunc (src/pert.cpp:59-136) with pert::x, pert::y
double pert_xy(const PertSpec& q, double a, double b, double c, double d, int i, int j) {
    const double eps = 1.e-14;
    double xval, yval, xyval = 0.;
    auto X = [&]() { return b * (double)i + a; };
    auto Y = [&]() { return d * (double)j + c; };
    switch (q.type) {
        case 0:
            xyval = 1.;
            break;
        case 1: {
            if (q.dx < eps) {
                xval = 0.;
            } else {
                double u = (X() - q.x0) / q.dx;
                xval = u * u;
            }
            if (q.dy < eps) {
                yval = 0.;
            } else {
                double u = (Y() - q.y0) / q.dy;
                yval = u * u;
            }
            xyval = std::exp(-xval - yval);
            break;
        }
        case 2: {
            if (q.dx < eps) {
                xval = 0.;
            } else {
                double u = (X() - q.x0) / q.dx;
                xval = u * u;
            }
            if (q.dy < eps) {
                yval = 0.;
            } else {
                double u = (Y() - q.y0) / q.dy;
                yval = u * u;
            }
            if (xval + yval <= 1.) xyval = 1.;
            break;
        }
        case 3:
            xval = (q.dx < eps) ? 1 : X() / q.dx + q.x0;
            yval = (q.dy < eps) ? 1 : Y() / q.dy + q.y0;
            xyval = xval * yval;
            break;
        case 4:
            if (q.dx < eps)
                xval = 1.;
            else if (std::fabs(std::fabs(X() - q.x0) - q.dx) < eps)
                xval = 0.5;
            else if (std::fabs(X() - q.x0) < q.dx)
                xval = 1.;
            else
                xval = 0.;
            if (q.dy < eps)
                yval = 1.;
            else if (std::fabs(std::fabs(Y() - q.y0) - q.dy) < eps)
                yval = 0.5;
            else if (std::fabs(Y() - q.y0) < q.dy)
                yval = 1.;
            else
                yval = 0.;
            xyval = xval * yval;
            break;
    }
    return xyval;
}

}  // namespace

void* Solver::dalloc(size_t bytes) {
    void* p = nullptr;
    cuda_check(cudaMalloc(&p, bytes ? bytes : 8), "cudaMalloc");
    cuda_check(cudaMemsetAsync(p, 0, bytes ? bytes : 8, stream_), "cudaMemset");
    owned_.push_back(p);
    return p;
}

double* Solver::scratch(size_t n) {
    if (n > scratch_n_) {
        if (scratch_) cudaFree(scratch_);
        cuda_check(cudaMalloc(&scratch_, n * sizeof(double)), "cudaMalloc scratch");
        scratch_n_ = n;
    }
    return scratch_;
}

Solver::Solver(const std::string& infile, int precision, int device) : precision_(precision), device_(device) {
    if (precision != 0 && precision != 1) throw std::runtime_error("precision must be 0 (FP64) or 1 (FP32)");
    P_ = read_problem(infile);
    cuda_check(cudaSetDevice(device), "cudaSetDevice");
    // reserve the allocation-free read-back buffer on this device now (the
    // lookup loads its module, which lazy module loading would otherwise
    // defer to the first fdf_get_field_noalloc call)
    noalloc_field_buffer(device);
    cuda_check(cudaStreamCreateWithFlags(&stream_, cudaStreamNonBlocking), "cudaStreamCreate");
    own_stream_ = stream_;
    // RK coefficients: src/rk.cpp:8-98
    switch (P_.rkorder) {
        case 1:
            nstages_ = 1;
            A_[0] = 0.; B_[0] = 1.; C_[0] = 0.; C_[1] = 1.;
            break;
        case 2:
            nstages_ = 2;
            A_[0] = 0.; A_[1] = -1.; B_[0] = 1.; B_[1] = 0.5;
            C_[0] = 0.; C_[1] = 1.; C_[2] = 1.;
            break;
        case 3:
            nstages_ = 3;
            A_[0] = 0.; A_[1] = -5. / 9.; A_[2] = -153. / 128.;
            B_[0] = 1. / 3.; B_[1] = 15. / 16.; B_[2] = 8. / 15.;
            C_[0] = 0.; C_[1] = 1. / 3.; C_[2] = 3. / 4.; C_[3] = 1.;
            break;
        case 4:
            nstages_ = 5;
            A_[0] = 0.;
            A_[1] = -567301805773. / 1357537059087.;
            A_[2] = -2404267990393. / 2016746695238.;
            A_[3] = -3550918686646. / 2091501179385.;
            A_[4] = -1275806237668. / 842570457699.;
            B_[0] = 1432997174477. / 9575080441755.;
            B_[1] = 5161836677717. / 13612068292357.;
            B_[2] = 1720146321549. / 2090206949498.;
            B_[3] = 3134564353537. / 4481467310338.;
            B_[4] = 2277821191437. / 14882151754819.;
            C_[0] = 0.;
            C_[1] = 1432997174477. / 9575080441755.;
            C_[2] = 2526269341429. / 6820363962896.;
            C_[3] = 2006345519317. / 3224310063776.;
            C_[4] = 2802321613138. / 2924317926251.;
            C_[5] = 1.;
            break;
        default:
            throw std::runtime_error("Error in initializing RK method");
    }
    // layout and field bookkeeping: src/fields.cpp:53-142
    L_.ndim = P_.ndim;
    L_.mode = P_.mode;
    for (int i = 0; i < 3; i++) L_.nx[i] = P_.nx[i];
    if (P_.ndim == 3) {
        long long nzp = ((P_.nx[2] + FDF_PITCH_ALIGN - 1) / FDF_PITCH_ALIGN) * FDF_PITCH_ALIGN;
        L_.s2 = 1;
        L_.s1 = nzp;
        L_.s0 = (long long)P_.nx[1] * nzp;
    } else {
        long long nyp = ((P_.nx[1] + FDF_PITCH_ALIGN - 1) / FDF_PITCH_ALIGN) * FDF_PITCH_ALIGN;
        L_.s2 = 0;
        L_.s1 = 1;
        L_.s0 = nyp;
    }
    L_.cstride = (long long)P_.nx[0] * L_.s0;
    // keep component starts 256-byte aligned
    L_.cstride = ((L_.cstride + 31) / 32) * 32;
    int nfields = (P_.ndim == 3) ? 9 : (P_.mode == 2 ? 5 : 3);
    int nfieldsp = 0;
    if (P_.plastic()) {
        nfieldsp = P_.plastic_tensor ? 8 : 2;
        if (P_.ndim == 2 && P_.mode == 2) nfields = 6;
    }
    L_.nfields = nfields;
    L_.nfieldsp = nfieldsp;
    if (P_.ndim == 3) {
        L_.nv = 3;
        L_.ns = 6;
        for (int i = 0; i < 6; i++) L_.sidx[i] = i;
    } else if (P_.mode == 2) {
        L_.nv = 2;
        L_.ns = P_.plastic() ? 4 : 3;
        L_.sidx[0] = 0;
        L_.sidx[1] = 1;
        L_.sidx[2] = 3;
        L_.sidx[3] = 5;
    } else {
        L_.nv = 1;
        L_.ns = 2;
        L_.sidx[0] = 2;
        L_.sidx[1] = 4;
    }
    status_ = static_cast<int*>(dalloc(sizeof(int)));
    setup_geometry();
    setup_plastic_visits(setup_material());
    setup_boundaries();
    set_time_step();
    set_block_coefficients();
    if (precision_ == 0)
        init_fields<double>();
    else
        init_fields<float>();
    setup_interfaces();
    initial_interface_solve();
    // initial output on absolute stress and back (problem.cpp:74-78): part of
    // the reference's arithmetic in the FP64 path
    if (precision_ == 0) launch_stress_roundtrip<double>(L_, (double*)F_[cur_], S_, P_.s0, stream_);
    // initial front values at t = 0 (problem.cpp:82)
    if (P_.front_on && P_.front_field == "V")
        for (auto& I : ifaces_)
            if (I.kind >= 1) launch_front(I, 0., P_.front_value, stream_);
    blocks_dev_ = static_cast<BlockDev*>(dalloc(blocks_.size() * sizeof(BlockDev)));
    cuda_check(cudaMemcpyAsync(blocks_dev_, blocks_.data(), blocks_.size() * sizeof(BlockDev), cudaMemcpyHostToDevice,
                               stream_),
               "block table");
    cuda_check(cudaStreamSynchronize(stream_), "set-up");
    if (int st = check_status()) throw std::runtime_error("set-up failed with status " + std::to_string(st));
}

Solver::~Solver() {
    if (stream_) cudaStreamSynchronize(stream_);
    if (own_stream_ && own_stream_ != stream_) cudaStreamSynchronize(own_stream_);
    if (copy_stream_) {
        cudaStreamSynchronize(copy_stream_);
        cudaStreamDestroy(copy_stream_);
    }
    for (auto& r : ring_busy_) cudaEventDestroy(r.done);
    for (auto e : ring_events_) cudaEventDestroy(e);
    if (ring_) cudaFree(ring_);
    out_.reset();
    for (void* p : owned_) cudaFree(p);
    for (void* p : {F_[0], F_[1], DF_, FP_, M_, J_, (void*)M64_, (void*)J64_, (void*)X_, (void*)S_, (void*)ABS_,
                    (void*)scratch_, (void*)mat_, (void*)pmask_})
        if (p) cudaFree(p);
    for (auto g : graph_exec_)
        if (g) cudaGraphExecDestroy(g);
    free_staged_maps(staged_maps_);
    free_reg_maps(reg_maps_);
    if (step_dev_) cudaFree(step_dev_);
    if (energy_dev_) cudaFree(energy_dev_);
    if (stz_mu_prev_) cudaFree(stz_mu_prev_);
    mlp_free(mlp_);
    if (stz_counts_) cudaFree(stz_counts_);
    if (samples_) cudaFree(samples_);
    if (nsamples_) cudaFree(nsamples_);
    for (auto e : ev_pool_) cudaEventDestroy(e);
    for (auto& pe : ev_pending_) {
        cudaEventDestroy(pe.second.first);
        cudaEventDestroy(pe.second.second);
    }
    if (own_stream_) cudaStreamDestroy(own_stream_);
}

// block geometry: block.cpp:183-246 (surfaces), 769-1046 (grid, metrics)
void Solver::setup_geometry() {
    const int ndim = P_.ndim;
    const size_t cs = (size_t)L_.cstride;
    cuda_check(cudaMalloc(&X_, cs * ndim * sizeof(double)), "cudaMalloc x");
    cuda_check(cudaMalloc(&M64_, cs * ndim * ndim * sizeof(double)), "cudaMalloc metric");
    cuda_check(cudaMalloc(&J64_, cs * sizeof(double)), "cudaMalloc jac");
    cuda_check(cudaMemsetAsync(X_, 0, cs * ndim * sizeof(double), stream_), "memset");
    cuda_check(cudaMemsetAsync(M64_, 0, cs * ndim * ndim * sizeof(double), stream_), "memset");
    cuda_check(cudaMemsetAsync(J64_, 0, cs * sizeof(double), stream_), "memset");
    blocks_.resize(P_.blocks.size());
    std::vector<double*> surf_dev;
    for (size_t bi = 0; bi < P_.blocks.size(); bi++) {
        const BlockSpec& bs = P_.blocks[bi];
        BlockDev& B = blocks_[bi];
        std::memset(&B, 0, sizeof(B));
        GeoBlock g{};
        for (int d = 0; d < 3; d++) {
            B.lo[d] = bs.xm[d];
            B.n[d] = bs.nx[d];
            B.dx[d] = 1. / (double)(bs.nx[d] - 1);
            g.lo[d] = B.lo[d];
            g.n[d] = B.n[d];
            g.dx[d] = B.dx[d];
        }
        B.xb = 0;
        B.xe = B.n[0];
        for (int f = 0; f < 2 * ndim; f++) {
            int d = f / 2, o0, o1;
            other_dims(d, o0, o1);
            int n0 = bs.nx[o0], n1 = bs.nx[o1];
            size_t nn = (size_t)n0 * n1;
            std::vector<double> sx((size_t)ndim * nn, 0.);
            if (bs.bfile[f] != "none") {
                sx = read_doubles(bs.bfile[f], (size_t)ndim * nn, 0);
            } else {
                // flat surface: surface.cpp:55-101 with the corner/lengths of block.cpp:183-213
                double xin[3] = {bs.xb[0], bs.xb[1], bs.xb[2]};
                if (f % 2 == 1) xin[d] = bs.xb[d] + bs.lb[d];
                double l0 = bs.lb[o0], l1 = bs.lb[o1];
                for (int j = 0; j < n0; j++)
                    for (int k = 0; k < n1; k++) {
                        sx[(size_t)d * nn + (size_t)j * n1 + k] = xin[d];
                        sx[(size_t)o0 * nn + (size_t)j * n1 + k] = xin[o0] + l0 * (double)(j) / (double)(n0 - 1);
                        if (ndim == 3)
                            sx[(size_t)o1 * nn + (size_t)j * n1 + k] = xin[o1] + l1 * (double)(k) / (double)(n1 - 1);
                    }
            }
            double* dp = nullptr;
            cuda_check(cudaMalloc(&dp, sx.size() * sizeof(double)), "cudaMalloc surface");
            cuda_check(cudaMemcpyAsync(dp, sx.data(), sx.size() * sizeof(double), cudaMemcpyHostToDevice, stream_),
                       "upload surface");
            cuda_check(cudaStreamSynchronize(stream_), "upload surface");
            surf_dev.push_back(dp);
            g.surf[f] = dp;
            g.sn0[f] = n0;
            g.sn1[f] = n1;
        }
        launch_transfinite(L_, g, X_, stream_);
        launch_metrics(L_, g, P_.sbporder, X_, M64_, J64_, status_, stream_);
        cuda_check(cudaGetLastError(), "geometry kernels");
    }
    cuda_check(cudaStreamSynchronize(stream_), "geometry");
    for (double* p : surf_dev) cudaFree(p);
    if (check_status() & FDF_ERR_JACOBIAN) throw std::runtime_error("jacobian must be positive: grid is not smooth enough");
}

// heterogeneous material: fields::read_mat (src/fields.cpp:582-711). The file
// holds rho, lambda and G over the whole grid (C order, FP64, one array after
// the other); every value must be positive (fields.cpp:648). The planes stay
// FP64 in both precisions and are shared by all blocks.
std::vector<double> Solver::setup_material() {
    if (P_.matfile == "none") return {};
    const size_t n = (size_t)P_.nx[0] * P_.nx[1] * P_.nx[2];
    const int nmat = 3;
    std::vector<double> h = read_doubles(P_.matfile, (size_t)nmat * n, 0);
    for (size_t q = 0; q < h.size(); q++)
        if (!(h[q] > 0.) || !std::isfinite(h[q]))
            throw std::runtime_error("material properties must be positive and finite (" + P_.matfile + ", value " +
                                     std::to_string(q) + ")");
    const size_t cs = (size_t)L_.cstride;
    cuda_check(cudaMalloc(&mat_, cs * nmat * sizeof(double)), "cudaMalloc material");
    cuda_check(cudaMemsetAsync(mat_, 0, cs * nmat * sizeof(double), stream_), "memset");
    double* tmp = scratch(n);
    for (int c = 0; c < nmat; c++) {
        cuda_check(cudaMemcpyAsync(tmp, h.data() + c * n, n * sizeof(double), cudaMemcpyHostToDevice, stream_),
                   "upload material");
        launch_store_component<double>(L_, mat_, c, tmp, stream_);
        cuda_check(cudaStreamSynchronize(stream_), "upload material");
    }
    for (auto& B : blocks_) {
        B.mat = mat_;
        B.matstride = L_.cstride;
    }
    return h;
}

// the nodes block::calc_plastic reaches (block.cpp:442-589).  Its z loop
// index is also where it stores the bulk modulus K = lambda + 2/3 G, so after
// the first node of a column it continues at trunc(K) + 1: in 2D that ends
// the column's only node; in 3D the loop leaves the block after the first z
// node when trunc(K) + 1 is past the block's last z node, visits the node
// trunc(K) + 1 when it is inside the block (with a heterogeneous material a
// chain of nodes), and never ends when a chain comes back to a node.
void Solver::setup_plastic_visits(const std::vector<double>& mat) {
    pvisit_ref_ = 0;
    if (!P_.plastic() || P_.ndim != 3) {
        apply_plastic_rule();
        return;
    }
    const size_t n = (size_t)P_.nx[0] * P_.nx[1] * P_.nx[2];
    const int ny = P_.nx[1], nz = P_.nx[2];
    std::vector<long long> extra;   // nodes reached beyond the first of a column
    for (size_t bi = 0; bi < blocks_.size() && plastic_stuck_.empty(); bi++) {
        const BlockDev& B = blocks_[bi];
        const BlockSpec& bs = P_.blocks[bi];
        const int lo2 = B.lo[2], hi2 = B.lo[2] + B.n[2];
        for (int i = B.lo[0]; i < B.lo[0] + B.n[0] && plastic_stuck_.empty(); i++)
            for (int j = B.lo[1]; j < B.lo[1] + B.n[1] && plastic_stuck_.empty(); j++) {
                int visits = 0;
                for (int k = lo2; k < hi2;) {
                    if (k < lo2 || ++visits > nz + 1) {
                        plastic_stuck_ = k < lo2 ? "the reference's plastic update (block.cpp:451-524) reaches nodes "
                                                   "outside their block for this problem"
                                                 : "the reference's plastic update (block.cpp:451-524) does not "
                                                   "terminate for this problem: its z loop index is overwritten by "
                                                   "the bulk modulus lambda + 2/3 G";
                        break;
                    }
                    const size_t q = ((size_t)i * ny + j) * nz + k;
                    const double K = mat.empty() ? bs.lam + 2. / 3. * bs.g : mat[n + q] + 2. / 3. * mat[2 * n + q];
                    if (!(K < 2147483647.)) {
                        plastic_stuck_ = "the bulk modulus lambda + 2/3 G does not fit the reference's int loop index";
                        break;
                    }
                    if (k != lo2) extra.push_back((long long)i * L_.s0 + (long long)j * L_.s1 + k);
                    k = (int)K + 1;
                }
            }
    }
    pvisit_ref_ = extra.empty() ? 1 : 2;
    if (pvisit_ref_ == 2 && plastic_stuck_.empty()) {
        std::vector<unsigned char> m((size_t)L_.cstride, 0);
        for (const auto& B : blocks_)
            for (int i = B.lo[0]; i < B.lo[0] + B.n[0]; i++)
                for (int j = B.lo[1]; j < B.lo[1] + B.n[1]; j++)
                    m[(size_t)i * L_.s0 + (size_t)j * L_.s1 + B.lo[2]] = 1;
        for (long long q : extra) m[(size_t)q] = 1;
        cuda_check(cudaMalloc(&pmask_, m.size()), "cudaMalloc plastic mask");
        cuda_check(cudaMemcpy(pmask_, m.data(), m.size(), cudaMemcpyHostToDevice), "upload plastic mask");
    }
    apply_plastic_rule();
}

void Solver::apply_plastic_rule() {
    for (auto& B : blocks_) {
        B.ptrunc = plastic_rule_ == 0 ? 1 : 0;
        B.pvisit = plastic_rule_ == 0 ? pvisit_ref_ : 0;
        B.pmask = pmask_;
    }
}

void Solver::check_plastic_rule() const {
    if (P_.plastic() && plastic_rule_ == 0 && !plastic_stuck_.empty())
        throw std::runtime_error(plastic_stuck_ + "; select the every-node rule (fdf_set_plastic_rule) to step it");
}

void Solver::set_plastic_rule(int rule) {
    if (rule != 0 && rule != 1) throw std::invalid_argument("plastic rule must be 0 (reference) or 1 (every node)");
    synchronize();
    plastic_rule_ = rule;
    apply_plastic_rule();
    cuda_check(cudaMemcpyAsync(blocks_dev_, blocks_.data(), blocks_.size() * sizeof(BlockDev), cudaMemcpyHostToDevice,
                               stream_),
               "block table");
    cuda_check(cudaStreamSynchronize(stream_), "block table");
    graph_dirty_ = true;
}

// boundary::boundary + allocate_normals: src/boundary.cpp:15-240
void Solver::setup_boundaries() {
    const int ndim = P_.ndim;
    const double h0 = sbp_h0(P_.sbporder);
    for (size_t bi = 0; bi < P_.blocks.size(); bi++) {
        const BlockSpec& bs = P_.blocks[bi];
        BlockDev& B = blocks_[bi];
        B.rho = bs.rho;
        B.lam = bs.lam;
        B.g = bs.g;
        B.cs = std::sqrt(bs.g / bs.rho);
        B.cp = std::sqrt((bs.lam + 2. * bs.g) / bs.rho);
        B.zs = bs.rho * B.cs;
        B.zp = bs.rho * B.cp;
        B.gamma = 1. - 2. * ((B.cs / B.cp) * (B.cs / B.cp));
        B.mu = bs.mu;
        B.coh = bs.coh;
        B.beta = bs.beta;
        B.eta = bs.eta;
        B.nu = 0.5 * bs.lam / (bs.lam + bs.g);
        for (int f = 0; f < 2 * ndim; f++) {
            const std::string& bt = bs.btype[f];
            B.bactive[f] = bt != "none";
            if (!B.bactive[f]) continue;
            if (bt == "absorbing") {
                B.r[f] = 0.; B.alpha[f] = 2.; B.theta[f] = 0.;
            } else if (bt == "free") {
                B.r[f] = -1.; B.alpha[f] = 1.; B.theta[f] = 0.;
            } else {
                B.r[f] = 1.; B.alpha[f] = 0.; B.theta[f] = 1.;
            }
            int d = f / 2, o0, o1;
            other_dims(d, o0, o1);
            int n0 = B.n[o0], n1 = B.n[o1];
            size_t nn = (size_t)n0 * n1;
            double* nx[3] = {nullptr, nullptr, nullptr};
            for (int k = 0; k < ndim; k++) nx[k] = (double*)dalloc(nn * sizeof(double));
            double* dl = (double*)dalloc(nn * sizeof(double));
            int at = (f % 2 == 0) ? B.lo[d] : B.lo[d] + B.n[d] - 1;
            launch_face_normals(L_, d, at, B.lo[o0], n0, B.lo[o1], n1, f % 2 == 0, h0 * B.dx[d], M64_, nx, dl, nullptr,
                                0, 0., stream_);
            for (int k = 0; k < 3; k++) B.fnx[f][k] = nx[k];
            B.fdl[f] = dl;
            B.fn1[f] = n1;
        }
    }
    cuda_check(cudaGetLastError(), "boundary normals");
}

// problem::set_time_step (src/problem.cpp:94-134) with block::get_min_dx
void Solver::set_time_step() {
    unsigned long long* dmax = (unsigned long long*)dalloc(sizeof(unsigned long long));
    for (size_t bi = 0; bi < blocks_.size(); bi++) {
        const BlockDev& B = blocks_[bi];
        GeoBlock g{};
        for (int d = 0; d < 3; d++) {
            g.lo[d] = B.lo[d];
            g.n[d] = B.n[d];
            g.dx[d] = B.dx[d];
        }
        launch_max_speed(L_, g, B.cs, M64_, mat_, dmax, stream_);
    }
    unsigned long long bits = 0;
    cuda_check(cudaMemcpyAsync(&bits, dmax, sizeof(bits), cudaMemcpyDeviceToHost, stream_), "min dx");
    cuda_check(cudaStreamSynchronize(stream_), "min dx");
    double vmax;
    std::memcpy(&vmax, &bits, sizeof(vmax));
    double dx = 1. / vmax;
    if (!(dx > 1.e-14)) throw std::runtime_error("a block does not have any grid spacing values");
    dt_ = P_.dt;
    cfl_ = P_.cfl;
    ttot_ = P_.ttot;
    nt_ = P_.nt;
    if ((ttot_ > 0. && nt_ > 0) && (dt_ == 0 && cfl_ == 0.)) {
        dt_ = ttot_ / (double)nt_;
        cfl_ = dt_ / dx;
    } else {
        if (dt_ > 0.)
            cfl_ = dt_ / dx;
        else
            dt_ = cfl_ * dx;
        if (ttot_ > 0.) {
            nt_ = (int)std::ceil(ttot_ / dt_);
            ttot_ = (double)nt_ * dt_;
        } else {
            ttot_ = (double)nt_ * dt_;
        }
    }
}

// stencil scale factors as calc_df forms them (block.cpp:1054-1055,
// 1166-1169, 1883-1886): dt/rho/dx0, then multiplied by dx0/dx1 and dx1/dx2
void Solver::set_block_coefficients() {
    for (auto& B : blocks_) {
        double invrho = dt_ / B.rho / B.dx[0];
        double g2lam = dt_ * (2. * B.g + B.lam) / B.dx[0];
        double g = dt_ * B.g / B.dx[0];
        double lambda = dt_ * B.lam / B.dx[0];
        for (int d = 0; d < P_.ndim; d++) {
            if (d > 0) {
                invrho *= B.dx[d - 1] / B.dx[d];
                g2lam *= B.dx[d - 1] / B.dx[d];
                g *= B.dx[d - 1] / B.dx[d];
                lambda *= B.dx[d - 1] / B.dx[d];
            }
            B.coef[d][0] = invrho;
            B.coef[d][1] = g2lam;
            B.coef[d][2] = g;
            B.coef[d][3] = lambda;
        }
    }
}

template <typename T>
void Solver::init_fields() {
    const size_t cs = (size_t)L_.cstride;
    for (int i = 0; i < 2; i++) {
        cuda_check(cudaMalloc(&F_[i], cs * L_.nfields * sizeof(T)), "cudaMalloc fields");
        cuda_check(cudaMemsetAsync(F_[i], 0, cs * L_.nfields * sizeof(T), stream_), "memset");
    }
    cuda_check(cudaMalloc(&DF_, cs * L_.nfields * sizeof(T)), "cudaMalloc rates");
    cuda_check(cudaMemsetAsync(DF_, 0, cs * L_.nfields * sizeof(T), stream_), "memset");
    if (L_.nfieldsp) {
        cuda_check(cudaMalloc(&FP_, cs * L_.nfieldsp * sizeof(T)), "cudaMalloc plastic fields");
        cuda_check(cudaMemsetAsync(FP_, 0, cs * L_.nfieldsp * sizeof(T), stream_), "memset");
    }
    if (sizeof(T) == 8) {
        M_ = M64_;
        J_ = J64_;
        M64_ = nullptr;
        J64_ = nullptr;
    } else {
        const size_t nm = cs * P_.ndim * P_.ndim;
        cuda_check(cudaMalloc(&M_, nm * sizeof(float)), "cudaMalloc metric32");
        cuda_check(cudaMalloc(&J_, cs * sizeof(float)), "cudaMalloc jac32");
        launch_to_float(M64_, (float*)M_, (long long)nm, stream_);
        launch_to_float(J64_, (float*)J_, (long long)cs, stream_);
    }
    if (P_.loadfile != "none") {
        // heterogeneous initial stress: fields.cpp:452-580 (ns arrays over the whole grid)
        const size_t n = (size_t)P_.nx[0] * P_.nx[1] * P_.nx[2];
        std::vector<double> h = read_doubles(P_.loadfile, (size_t)L_.ns * n, 0);
        cuda_check(cudaMalloc(&S_, cs * L_.ns * sizeof(double)), "cudaMalloc stress");
        cuda_check(cudaMemsetAsync(S_, 0, cs * L_.ns * sizeof(double), stream_), "memset");
        double* tmp = scratch(n);
        for (int c = 0; c < L_.ns; c++) {
            cuda_check(cudaMemcpyAsync(tmp, h.data() + c * n, n * sizeof(double), cudaMemcpyHostToDevice, stream_),
                       "upload stress");
            Layout Ls = L_;
            launch_store_component<double>(Ls, S_, c, tmp, stream_);
        }
        cuda_check(cudaStreamSynchronize(stream_), "upload stress");
    }
    cuda_check(cudaGetLastError(), "init fields");
}

// interface::interface, friction::friction, slipweak::slipweak, stz::stz
// (src/interface.cpp:17-534, src/friction.cpp:19-227, src/slipweak.cpp:19-182,
// src/stz.cpp:19-232)
void Solver::setup_interfaces() {
    const int ndim = P_.ndim;
    const double h0 = sbp_h0(P_.sbporder);
    const int nb1 = P_.nblocks[1], nb2 = P_.nblocks[2];
    std::unordered_map<long long, int> last_touch;
    ifaces_.resize(P_.ifaces.size());
    for (size_t n = 0; n < P_.ifaces.size(); n++) {
        const IfaceSpec& S = P_.ifaces[n];
        IfaceDev& I = ifaces_[n];
        std::memset(&I, 0, sizeof(I));
        I.kind = (S.kind == "locked") ? 0 : (S.kind == "frictionless") ? 1 : (S.kind == "slipweak") ? 2 : 3;
        I.direction = S.direction;
        const int D = S.direction;
        I.b1 = (S.idx1[0] * nb1 + S.idx1[1]) * nb2 + S.idx1[2];
        I.b2 = (S.idx2[0] * nb1 + S.idx2[1]) * nb2 + S.idx2[2];
        BlockDev& B1 = blocks_[I.b1];
        BlockDev& B2 = blocks_[I.b2];
        const BlockSpec& s1 = P_.blocks[I.b1];
        const BlockSpec& s2 = P_.blocks[I.b2];
        int o0, o1;
        other_dims(D, o0, o1);
        if (s1.nx[o0] != s2.nx[o0] || s1.nx[o1] != s2.nx[o1])
            throw std::runtime_error("interface blocks have different face sizes");
        I.n0 = s1.nx[o0];
        I.n1 = s1.nx[o1];
        for (int i = 0; i < 3; i++) I.mlb[i] = B1.lo[i];
        I.mlb[D] = B1.lo[D] + B1.n[D] - 1;
        B1.defer[2 * D + 1] = 1;
        B2.defer[2 * D] = 1;
        I.cp1 = B1.cp; I.cs1 = B1.cs; I.zp1 = B1.zp; I.zs1 = B1.zs;
        I.cp2 = B2.cp; I.cs2 = B2.cs; I.zp2 = B2.zp; I.zs2 = B2.zs;
        I.gamma1 = 1. - 2. * ((I.cs1 / I.cp1) * (I.cs1 / I.cp1));
        I.gamma2 = 1. - 2. * ((I.cs2 / I.cp2) * (I.cs2 / I.cp2));
        const size_t nn = (size_t)I.n0 * I.n1;
        // edge check (interface.cpp:331-347) on the two coordinate planes
        {
            std::vector<double> xa(nn), xb(nn);
            double* tmp = scratch(2 * nn);
            for (int c = 0; c < ndim; c++) {
                // gather both planes with a fetch of the whole component would be large; copy row by row
                for (int a = 0; a < I.n0; a++)
                    for (int side = 0; side < 2; side++) {
                        int pos[3] = {I.mlb[0], I.mlb[1], I.mlb[2]};
                        pos[o0] += a;
                        pos[D] += side;
                        long long id = pos[0] * L_.s0 + pos[1] * L_.s1 + pos[2] * L_.s2;
                        long long step = (o1 == 2) ? L_.s2 : L_.s1;
                        if (I.n1 == 1 || step == 1) {
                            cuda_check(cudaMemcpyAsync(tmp + side * nn + (size_t)a * I.n1, X_ + c * L_.cstride + id,
                                                       (size_t)I.n1 * sizeof(double), cudaMemcpyDeviceToDevice, stream_),
                                       "gather plane");
                        } else {
                            cuda_check(cudaMemcpy2DAsync(tmp + side * nn + (size_t)a * I.n1, sizeof(double),
                                                         X_ + c * L_.cstride + id, step * sizeof(double),
                                                         sizeof(double), I.n1, cudaMemcpyDeviceToDevice, stream_),
                                       "gather plane");
                        }
                    }
                cuda_check(cudaMemcpyAsync(xa.data(), tmp, nn * sizeof(double), cudaMemcpyDeviceToHost, stream_), "d2h");
                cuda_check(cudaMemcpyAsync(xb.data(), tmp + nn, nn * sizeof(double), cudaMemcpyDeviceToHost, stream_),
                           "d2h");
                cuda_check(cudaStreamSynchronize(stream_), "edge check");
                for (size_t m = 0; m < nn; m++)
                    if (!(std::fabs(xa[m] - xb[m]) <= (1.e-8 + 1.e-5 * std::fabs(xb[m]))))
                        throw std::runtime_error("interface " + std::to_string(n) + ": block edges do not match");
            }
        }
        double* nx[3] = {nullptr, nullptr, nullptr};
        for (int k = 0; k < ndim; k++) nx[k] = (double*)dalloc(nn * sizeof(double));
        double* dl1 = (double*)dalloc(nn * sizeof(double));
        double* dl2 = (double*)dalloc(nn * sizeof(double));
        launch_face_normals(L_, D, I.mlb[D], I.mlb[o0], I.n0, I.mlb[o1], I.n1, 0, h0 * B1.dx[D], M64_ ? M64_ : (double*)M_,
                            nx, dl1, dl2, I.mlb[D] + 1, h0 * B2.dx[D], stream_);
        for (int k = 0; k < 3; k++) I.nx[k] = nx[k];
        I.dl1 = dl1;
        I.dl2 = dl2;
        // finalisation flags: the last interface touching a node finishes it
        for (int side = 0; side < 2; side++)
            for (int a = 0; a < I.n0; a++)
                for (int b = 0; b < I.n1; b++) {
                    int pos[3] = {I.mlb[0], I.mlb[1], I.mlb[2]};
                    pos[o0] += a;
                    pos[o1] += b;
                    pos[D] += side;
                    long long key = ((long long)pos[0] * P_.nx[1] + pos[1]) * P_.nx[2] + pos[2];
                    last_touch[key] = (int)n;
                }
        if (I.kind >= 1) {
            const size_t nt = (size_t)(ndim - 1) * nn;
            I.u = (double*)dalloc(nn * 8); I.du = (double*)dalloc(nn * 8); I.v = (double*)dalloc(nn * 8);
            I.s = (double*)dalloc(nn * 8); I.sn = (double*)dalloc(nn * 8);
            I.ux = (double*)dalloc(nt * 8); I.dux = (double*)dalloc(nt * 8); I.vx = (double*)dalloc(nt * 8);
            I.sx = (double*)dalloc(nt * 8);
            I.tfront = (double*)dalloc(nn * 8);
            std::vector<double> minus1(nn, -1.);
            cuda_check(cudaMemcpyAsync(I.tfront, minus1.data(), nn * 8, cudaMemcpyHostToDevice, stream_), "front init");
            // perturbation coordinate map on the fault plane (friction.cpp:131-176, pert.cpp:7-73)
            double x2[2] = {s1.xb[o0], s1.xb[o1]}, l2[2] = {s1.lb[o0], s1.lb[o1]};
            int n2[2] = {I.n0, I.n1};
            const double pa = (double)(0) / (double)(n2[0] - 1) * l2[0] + x2[0];
            const double pb = l2[0] / (double)(n2[0] - 1);
            const double pc = (double)(0) / (double)(n2[1] - 1) * l2[1] + x2[1];
            const double pd = l2[1] / (double)(n2[1] - 1);
            auto make_perts = [&](const std::vector<PertSpec>& src, int nval) -> const PertDev* {
                std::vector<PertDev> h(src.size());
                for (size_t m = 0; m < src.size(); m++) {
                    PertDev& q = h[m];
                    std::memset(&q, 0, sizeof(q));
                    q.t0 = src[m].t0;
                    for (int k = 0; k < nval; k++) q.val[k] = src[m].val[k];
                    q.shaped = src[m].type != 0;
                    if (q.shaped) {
                        std::vector<double> xy(nn);
                        for (int a = 0; a < I.n0; a++)
                            for (int b = 0; b < I.n1; b++)
                                xy[(size_t)a * I.n1 + b] = pert_xy(src[m], pa, pb, pc, pd, a, b);
                        double* dp = (double*)dalloc(nn * 8);
                        cuda_check(cudaMemcpyAsync(dp, xy.data(), nn * 8, cudaMemcpyHostToDevice, stream_), "pert");
                        cuda_check(cudaStreamSynchronize(stream_), "pert");
                        q.xy = dp;
                    }
                }
                PertDev* dp = (PertDev*)dalloc(std::max<size_t>(1, h.size()) * sizeof(PertDev));
                if (!h.empty())
                    cuda_check(cudaMemcpyAsync(dp, h.data(), h.size() * sizeof(PertDev), cudaMemcpyHostToDevice, stream_),
                               "perts");
                cuda_check(cudaStreamSynchronize(stream_), "perts");
                return dp;
            };
            auto upload = [&](const std::vector<double>& v) -> double* {
                double* dp = (double*)dalloc(v.size() * 8);
                cuda_check(cudaMemcpyAsync(dp, v.data(), v.size() * 8, cudaMemcpyHostToDevice, stream_), "upload");
                cuda_check(cudaStreamSynchronize(stream_), "upload");
                return dp;
            };
            I.nloads = (int)S.loads.size();
            I.loads = make_perts(S.loads, 3);
            if (S.loadfile != "none") {
                I.load_file = 1;
                std::vector<double> s1v = read_doubles(S.loadfile, nn, 0), s2v = read_doubles(S.loadfile, nn, nn),
                                    s3v = read_doubles(S.loadfile, nn, 2 * nn);
                if (ndim == 2 && P_.mode == 2) std::fill(s3v.begin(), s3v.end(), 0.);
                if (ndim == 2 && P_.mode == 3) std::fill(s2v.begin(), s2v.end(), 0.);
                I.s1 = upload(s1v);
                I.s2 = upload(s2v);
                I.s3 = upload(s3v);
            }
            if (I.kind == 2 || I.kind == 3) {
                int npar = (I.kind == 2) ? 6 : 9;
                I.nperts = (int)S.perts.size();
                I.perts = make_perts(S.perts, npar);
                if (S.paramfile != "none") {
                    I.param_file = 1;
                    for (int k = 0; k < npar; k++) I.par[k] = upload(read_doubles(S.paramfile, nn, (size_t)k * nn));
                }
            }
            if (I.kind == 3) {
                std::vector<double> st(nn, 0.);
                if (S.statefile != "none") st = read_doubles(S.statefile, nn, 0);
                for (auto& v : st) v += S.chi0;
                I.state = upload(st);
                I.dstate = (double*)dalloc(nn * 8);
                I.dstatedt = (double*)dalloc(nn * 8);
            }
        }
    }
    for (size_t n = 0; n < ifaces_.size(); n++) {
        IfaceDev& I = ifaces_[n];
        const int D = I.direction;
        int o0, o1;
        other_dims(D, o0, o1);
        const size_t nn = (size_t)I.n0 * I.n1;
        std::vector<unsigned char> f1(nn), f2(nn);
        for (int side = 0; side < 2; side++)
            for (int a = 0; a < I.n0; a++)
                for (int b = 0; b < I.n1; b++) {
                    int pos[3] = {I.mlb[0], I.mlb[1], I.mlb[2]};
                    pos[o0] += a;
                    pos[o1] += b;
                    pos[D] += side;
                    long long key = ((long long)pos[0] * P_.nx[1] + pos[1]) * P_.nx[2] + pos[2];
                    (side ? f2 : f1)[(size_t)a * I.n1 + b] = last_touch[key] == (int)n;
                }
        unsigned char* d1 = (unsigned char*)dalloc(nn);
        unsigned char* d2 = (unsigned char*)dalloc(nn);
        cuda_check(cudaMemcpyAsync(d1, f1.data(), nn, cudaMemcpyHostToDevice, stream_), "flags");
        cuda_check(cudaMemcpyAsync(d2, f2.data(), nn, cudaMemcpyHostToDevice, stream_), "flags");
        cuda_check(cudaStreamSynchronize(stream_), "flags");
        I.fin1 = d1;
        I.fin2 = d2;
    }
    if (M64_) {
        cudaFree(M64_);
        cudaFree(J64_);
        M64_ = nullptr;
        J64_ = nullptr;
    }
    cuda_check(cudaGetLastError(), "interfaces");
}

// domain::domain calls apply_bcs(0., 0., f, true) on every interface (domain.cpp:141-143)
void Solver::initial_interface_solve() {
    StageArgs sa{};
    sa.dt = 0.;
    sa.t = 0.;
    for (auto& I : ifaces_) {
        if (I.kind < 1) continue;
        const BlockDev& B1 = blocks_[I.b1];
        const BlockDev& B2 = blocks_[I.b2];
        if (precision_ == 0) {
            IfaceArgs<double> a{};
            a.L = L_;
            std::memcpy(a.s0, P_.s0, sizeof(a.s0));
            a.F = (double*)F_[cur_];
            a.Fn = (double*)F_[cur_];
            a.DF = (double*)DF_;
            a.FP = (double*)FP_;
            a.S = S_;
            a.status = status_;
            launch_interface<double>(a, I, B1, B2, sa, 1, stream_);
        } else {
            IfaceArgs<float> a{};
            a.L = L_;
            std::memcpy(a.s0, P_.s0, sizeof(a.s0));
            a.F = (float*)F_[cur_];
            a.Fn = (float*)F_[cur_];
            a.DF = (float*)DF_;
            a.FP = (float*)FP_;
            a.S = S_;
            a.status = status_;
            launch_interface<float>(a, I, B1, B2, sa, 1, stream_);
        }
    }
    cuda_check(cudaGetLastError(), "initial interface solve");
}

cudaEvent_t Solver::ev_get() {
    if (!ev_pool_.empty()) {
        cudaEvent_t e = ev_pool_.back();
        ev_pool_.pop_back();
        return e;
    }
    cudaEvent_t e;
    cuda_check(cudaEventCreate(&e), "event");
    return e;
}

void Solver::prof_flush() {
    for (auto& pe : ev_pending_) {
        float ms = 0;
        cudaEventSynchronize(pe.second.second);
        cudaEventElapsedTime(&ms, pe.second.first, pe.second.second);
        prof_ms_[pe.first] += ms;
        prof_n_[pe.first] += 1;
        ev_pool_.push_back(pe.second.first);
        ev_pool_.push_back(pe.second.second);
    }
    ev_pending_.clear();
}

void Solver::set_profile(bool on) {
    prof_flush();
    profile_ = on;
    for (int i = 0; i < 4; i++) {
        prof_ms_[i] = 0;
        prof_n_[i] = 0;
    }
}

void Solver::profile_read(int kernel, double* total_ms, long long* launches) {
    prof_flush();
    *total_ms = prof_ms_[kernel & 3];
    *launches = prof_n_[kernel & 3];
}

int Solver::volume_kernel_active() const {
    // the marching kernels hold one material per block: heterogeneous
    // material runs the reference-order kernel
    if (vkernel_ == 0 || precision_ != 1 || mat_) return 0;
    if (L_.ndim == 2) {   // tiled 2D kernel (elastic, no dissipation; kinds 1 and 3) or none
        if ((vkernel_ != 1 && vkernel_ != 3) || P_.plastic() || P_.cdiss > 0.) return 0;
        for (auto& B : blocks_)
            if (!fast2d_supported(L_, B, P_.sbporder)) return 0;
        return 1;
    }
    for (auto& B : blocks_) {
        if (vkernel_ == 1 && !fast3d_supported(L_, B, P_.sbporder)) return 0;
        if (vkernel_ == 2 && !staged3d_supported(L_, B, P_.sbporder)) return 0;
        if (vkernel_ == 3 && !reg3d_supported(L_, B, P_.sbporder)) return 0;
    }
    return vkernel_;
}

bool Solver::fast_kernel_active() const { return volume_kernel_active() != 0; }

template <typename T>
void Solver::stage_impl(double dt, int stage, double t, bool for_step) {
    StageArgs sa{};
    sa.dt = dt;
    sa.A = A_[stage];
    sa.B = B_[stage];
    sa.t = t + C_[stage] * dt;
    sa.last = (stage + 1 == nstages_);
    sa.plastic = P_.plastic() ? 1 : 0;
    sa.roundtrip = (precision_ == 0 && for_step) ? 1 : 0;
    sa.abs_out = 0;
    sa.front_on = (for_step && P_.front_on && P_.front_field == "V") ? 1 : 0;
    sa.front_value = P_.front_value;
    sa.tfront = (double)(step_index_ + 1) * dt;
    sa.step_dev = capturing_ ? step_dev_ : nullptr;
    sa.cst = C_[stage];
    sa.wait_limit = wait_limit_;
    T* Fo = (T*)F_[cur_];
    T* Fn = (T*)F_[1 - cur_];
    VolumeArgs<T> va{};
    va.L = L_;
    va.order = P_.sbporder;
    va.cdiss = P_.cdiss;
    std::memcpy(va.s0, P_.s0, sizeof(va.s0));
    va.F = Fo;
    va.Fn = Fn;
    va.DF = (T*)DF_;
    va.M = (const T*)M_;
    va.J = (const T*)J_;
    va.FP = (T*)FP_;
    va.S = S_;
    va.ABS = (sa.roundtrip && sa.last) ? ABS_ : nullptr;
    va.plastic_tensor = P_.plastic_tensor ? 1 : 0;
    const int vk = volume_kernel_active();
    if (slab_ && vk != 0 && vk != 3)
        throw std::runtime_error("x slabs run the register-window (3) or reference-order (0) volume kernel");
    // the reference-order kernel takes every block in one launch
    const bool all_exact = (sizeof(T) == 8 || vk == 0) && (int)blocks_.size() <= FDF_ALLB_MAX;
    if (all_exact) {
        cudaEvent_t e0 = nullptr, e1 = nullptr;
        if (profile_) {
            e0 = ev_get();
            e1 = ev_get();
            cudaEventRecord(e0, stream_);
        }
        launch_volume_exact_all<T>(va, blocks_dev_, blocks_.data(), (int)blocks_.size(), sa, stream_);
        if (profile_) {
            cudaEventRecord(e1, stream_);
            ev_pending_.push_back({0, {e0, e1}});
        }
    }
    for (size_t b = 0; b < blocks_.size() && !all_exact; b++) {
        cudaEvent_t e0 = nullptr, e1 = nullptr;
        if (profile_) {
            e0 = ev_get();
            e1 = ev_get();
            cudaEventRecord(e0, stream_);
        }
        if constexpr (sizeof(T) == 4) {
            // register window: the pre-passes of up to FDF_ALLB_MAX blocks in one
            // launch, timed with the first of them
            if (vk == 3 && P_.cdiss <= 0. && b % FDF_ALLB_MAX == 0) {
                if (!reg_maps_)
                    reg_maps_ = make_reg_maps(L_, (const float*)F_[0], (const float*)F_[1], (const float*)M_,
                                              (const float*)J_, (const float*)DF_, blocks_.data(), (int)blocks_.size());
                const int nb = std::min<int>(FDF_ALLB_MAX, (int)(blocks_.size() - b));
                launch_prepass_reg3d(va, blocks_dev_, blocks_.data(), (int)b, nb, sa, reg_maps_, stream_);
            }
            if (vk == 2) {
                if (!staged_maps_)
                    staged_maps_ = make_staged_maps(L_, (const float*)F_[0], (const float*)F_[1], (const float*)M_,
                                                    (const float*)J_, P_.sbporder);
                launch_volume_staged3d(va, blocks_[b], sa, status_, staged_maps_, stream_);
            } else if (vk == 3) {
                if (!reg_maps_)
                    reg_maps_ = make_reg_maps(L_, (const float*)F_[0], (const float*)F_[1], (const float*)M_,
                                              (const float*)J_, (const float*)DF_, blocks_.data(), (int)blocks_.size());
                launch_volume_reg3d(va, blocks_[b], (int)b, sa, status_, reg_maps_, stream_);
            }
            else if (vk == 1 && L_.ndim == 3)
                launch_volume_fast3d(va, blocks_[b], sa, stream_);
            else if (vk == 1)
                launch_volume_fast2d(va, blocks_[b], sa, stream_);
            else
                launch_volume_exact<T>(va, blocks_[b], sa, stream_);
        } else {
            launch_volume_exact<T>(va, blocks_[b], sa, stream_);
        }
        if (profile_) {
            cudaEventRecord(e1, stream_);
            ev_pending_.push_back({0, {e0, e1}});
        }
    }
    IfaceArgs<T> ia{};
    ia.L = L_;
    std::memcpy(ia.s0, P_.s0, sizeof(ia.s0));
    ia.F = Fo;
    ia.Fn = Fn;
    ia.DF = (T*)DF_;
    ia.FP = (T*)FP_;
    ia.S = S_;
    ia.ABS = va.ABS;
    ia.plastic_tensor = va.plastic_tensor;
    ia.status = status_;
    cudaEvent_t e0 = nullptr, e1 = nullptr;
    if (profile_ && !ifaces_.empty()) {
        e0 = ev_get();
        e1 = ev_get();
        cudaEventRecord(e0, stream_);
    }
    for (auto& I : ifaces_) launch_interface<T>(ia, I, blocks_[I.b1], blocks_[I.b2], sa, 0, stream_);
    if (sa.last && sa.plastic)
        for (auto& I : ifaces_)
            if (I.kind >= 1) launch_interface<T>(ia, I, blocks_[I.b1], blocks_[I.b2], sa, 1, stream_);
    if (profile_ && !ifaces_.empty()) {
        cudaEventRecord(e1, stream_);
        ev_pending_.push_back({1, {e0, e1}});
    }
    cur_ = 1 - cur_;
}

void Solver::do_rk_stage(double dt, int stage, double t) {
    if (stage < 0 || stage >= nstages_) throw std::runtime_error("stage out of range");
    check_plastic_rule();
    if (precision_ == 0)
        stage_impl<double>(dt, stage, t, false);
    else
        stage_impl<float>(dt, stage, t, false);
    cuda_check(cudaGetLastError(), "stage launch");
}

void Solver::step_stage(int stage) {
    if (stage != stage_next_)
        throw std::runtime_error("step_stage: expected stage " + std::to_string(stage_next_) + ", got " +
                                 std::to_string(stage));
    check_plastic_rule();
    if (precision_ == 0)
        stage_impl<double>(dt_, stage, (double)step_index_ * dt_, true);
    else
        stage_impl<float>(dt_, stage, (double)step_index_ * dt_, true);
    cuda_check(cudaGetLastError(), "stage launch");
    stage_next_ = (stage + 1) % nstages_;
    if (stage_next_ == 0) step_index_++;
}

void Solver::set_x_range(int x0, int x1) {
    const int nx = P_.nx[0];
    if (x0 < 0 || x1 > nx || x0 >= x1) throw std::runtime_error("set_x_range: need 0 <= x0 < x1 <= nx");
    const bool whole = (x0 == 0 && x1 == nx);
    if (stage_next_ != 0) throw std::runtime_error("set_x_range: a step begun by step_stage is unfinished");
    if (!whole) {
        if (P_.ndim != 3) throw std::runtime_error("x slabs cover 3D problems");
        if (P_.cdiss > 0.) throw std::runtime_error("x slabs: artificial dissipation is not supported");
        const int vk = volume_kernel_active();
        if (precision_ == 1 && vk != 0 && vk != 3)
            throw std::runtime_error("x slabs run the register-window (3) or reference-order (0) volume kernel");
        if (out_) throw std::runtime_error("x slabs: output units are written by whole-domain runs");
        // a cut lies at least SLAB_MARGIN planes inside an x block: the closure
        // rows and x faces (and any x-normal interface) stay with one slab, and
        // a slab's first chunk starts past the closure rows
        constexpr int SLAB_MARGIN = 16;
        for (int c : {x0, x1}) {
            if (c == 0 || c == nx) continue;
            for (const auto& B : blocks_)
                if (c >= B.lo[0] && c < B.lo[0] + B.n[0] &&
                    (c - B.lo[0] < SLAB_MARGIN || B.lo[0] + B.n[0] - c < SLAB_MARGIN))
                    throw std::runtime_error("set_x_range: cut at x = " + std::to_string(c) +
                                             " is within 16 planes of an x block face");
        }
        // the planes packed for a neighbour lie inside the slab
        if (x1 - x0 < SLAB_MARGIN) throw std::runtime_error("set_x_range: a slab spans at least 16 planes");
    }
    synchronize();
    for (auto& B : blocks_) {
        B.xb = std::min(std::max(x0 - B.lo[0], 0), B.n[0]);
        B.xe = std::min(std::max(x1 - B.lo[0], 0), B.n[0]);
        if (B.xe < B.xb) B.xe = B.xb;
    }
    cuda_check(cudaMemcpyAsync(blocks_dev_, blocks_.data(), blocks_.size() * sizeof(BlockDev), cudaMemcpyHostToDevice,
                               stream_),
               "block table");
    cuda_check(cudaStreamSynchronize(stream_), "block table");
    slab_ = !whole;
    xr0_ = x0;
    xr1_ = x1;
    graph_dirty_ = true;
}

long long Solver::ghost_count() const { return (long long)L_.nfields * ghost_planes() * L_.s0; }

void Solver::pack_ghosts(int side, void* dst) {
    if (!slab_) throw std::runtime_error("pack_ghosts: no x slab set");
    if (side != 0 && side != 1) throw std::runtime_error("pack_ghosts: side is 0 or 1");
    if (side == 0 ? xr0_ == 0 : xr1_ == P_.nx[0]) throw std::runtime_error("pack_ghosts: no neighbour on that side");
    if (!dst) throw std::runtime_error("pack_ghosts: null buffer");
    const int g = ghost_planes();
    const long long off = (long long)(side == 0 ? xr0_ : xr1_ - g) * L_.s0;
    launch_ghost_copy(F_[cur_], precision_ == 0 ? 8 : 4, L_.cstride, L_.nfields, off, (long long)g * L_.s0, dst, 0,
                      stream_);
    cuda_check(cudaGetLastError(), "ghost pack");
}

void Solver::unpack_ghosts(int side, const void* src) {
    if (!slab_) throw std::runtime_error("unpack_ghosts: no x slab set");
    if (side != 0 && side != 1) throw std::runtime_error("unpack_ghosts: side is 0 or 1");
    if (side == 0 ? xr0_ == 0 : xr1_ == P_.nx[0]) throw std::runtime_error("unpack_ghosts: no neighbour on that side");
    if (!src) throw std::runtime_error("unpack_ghosts: null buffer");
    const int g = ghost_planes();
    const long long off = (long long)(side == 0 ? xr0_ - g : xr1_) * L_.s0;
    launch_ghost_copy(F_[cur_], precision_ == 0 ? 8 : 4, L_.cstride, L_.nfields, off, (long long)g * L_.s0,
                      const_cast<void*>(src), 1, stream_);
    cuda_check(cudaGetLastError(), "ghost unpack");
}

void Solver::set_stream(bool own, cudaStream_t s) {
    if (capturing_) throw std::runtime_error("set_stream: a capture is in progress");
    synchronize();
    stream_ = own ? own_stream_ : s;
}

void Solver::step(int nsteps) {
    if (slab_)
        throw std::runtime_error("an x slab steps one stage at a time (step_stage) with a ghost exchange after each");
    if (stage_next_ != 0) throw std::runtime_error("step: a step begun by step_stage is unfinished");
    check_plastic_rule();
    // steps replay the captured one-step graphs when nothing on the host has
    // to happen between steps (no output units, no per-launch profiling)
    if (graphs_ && !out_ && !profile_ && nsteps >= 1) {
        step_graph(nsteps);
        return;
    }
    step_launches(nsteps);
}

void Solver::step_graph(int nsteps) {
    if (graph_dirty_) {
        for (auto& g : graph_exec_)
            if (g) {
                cudaGraphExecDestroy(g);
                g = nullptr;
            }
        graph_dirty_ = false;
    }
    if (!step_dev_) cuda_check(cudaMalloc(&step_dev_, sizeof(int)), "cudaMalloc step counter");
    // a graph of one step bakes in which field buffer it reads first: one graph
    // per parity; an odd number of stages leaves the other buffer current
    const int flip = nstages_ & 1;
    for (int par = 0; par < 2; par++) {
        if (graph_exec_[par] || (par != cur_ && !flip)) continue;
        if (par != cur_ && nsteps < 2) continue;   // captured when first needed
        const int cur0 = cur_, idx0 = step_index_;
        cur_ = par;
        cuda_check(cudaStreamBeginCapture(stream_, cudaStreamCaptureModeRelaxed), "begin capture");
        capturing_ = true;
        // if a stage throws while the stream captures, end the capture, drop the
        // partial graph and put the handle's state back before the error leaves
        struct CaptureGuard {
            Solver& s;
            int cur0, idx0;
            bool armed = true;
            ~CaptureGuard() {
                if (!armed) return;
                cudaGraph_t partial = nullptr;
                cudaStreamEndCapture(s.stream_, &partial);
                if (partial) cudaGraphDestroy(partial);
                cudaGetLastError();
                s.capturing_ = false;
                s.cur_ = cur0;
                s.step_index_ = idx0;
            }
        } guard{*this, cur0, idx0};
        for (int st = 0; st < nstages_; st++) {
            if (precision_ == 0)
                stage_impl<double>(dt_, st, 0., true);
            else
                stage_impl<float>(dt_, st, 0., true);
        }
        launch_step_advance(step_dev_, stream_);
        guard.armed = false;
        capturing_ = false;
        cudaGraph_t g = nullptr;
        cuda_check(cudaStreamEndCapture(stream_, &g), "end capture");
        const cudaError_t ie = cudaGraphInstantiate(&graph_exec_[par], g, 0);
        cudaGraphDestroy(g);
        cur_ = cur0;
        step_index_ = idx0;
        cuda_check(ie, "graph instantiate");
    }
    launch_set_step(step_dev_, step_index_, stream_);
    for (int n = 0; n < nsteps; n++) {
        cuda_check(cudaGraphLaunch(graph_exec_[cur_], stream_), "graph launch");
        cur_ ^= flip;
    }
    step_index_ += nsteps;
}

void Solver::step_launches(int nsteps) {
    for (int n = 0; n < nsteps; n++) {
        for (int st = 0; st < nstages_; st++) {
            if (precision_ == 0)
                stage_impl<double>(dt_, st, (double)step_index_ * dt_, true);
            else
                stage_impl<float>(dt_, st, (double)step_index_ * dt_, true);
        }
        cuda_check(cudaGetLastError(), "step launch");
        step_index_++;
        if (out_) out_->write(step_index_);
    }
}

void Solver::fetch_output_component(int comp, int tstep, double* out) {
    const bool stress = comp >= L_.nv && comp < L_.nv + L_.ns;
    if (stress && precision_ == 0 && tstep > 0 && ABS_) {
        const size_t n = (size_t)P_.nx[0] * P_.nx[1] * P_.nx[2];
        double* tmp = scratch(n);
        launch_fetch_component<double>(L_, ABS_, comp - L_.nv, 0, P_.s0, nullptr, tmp, stream_);
        fetch_to(tmp, n * sizeof(double), out);
        return;
    }
    get_field(comp, true, out);
}

void Solver::solve() {
    if (slab_) throw std::runtime_error("solve runs the whole domain: set_x_range(0, nx) first");
    if (!out_) {
        out_.reset(new OutputList(*this));
        if (out_->needs_abs_stress() && !ABS_) {
            cuda_check(cudaMalloc(&ABS_, (size_t)L_.cstride * L_.ns * sizeof(double)), "cudaMalloc output staging");
            cuda_check(cudaMemsetAsync(ABS_, 0, (size_t)L_.cstride * L_.ns * sizeof(double), stream_), "memset");
        }
        out_->write(step_index_);
    }
    // the status word is read every 16 steps (a device-side error stops the
    // run within 16 steps of it), so output copies overlap the steps between
    while (step_index_ < nt_) {
        step(std::min(16, nt_ - step_index_));
        if (int st = check_status()) throw std::runtime_error("solver status " + std::to_string(st));
    }
    out_->close();
    cuda_check(cudaStreamSynchronize(stream_), "solve");
}

void Solver::synchronize() {
    cuda_check(cudaStreamSynchronize(stream_), "synchronize");
    if (copy_stream_) cuda_check(cudaStreamSynchronize(copy_stream_), "synchronize read-back");
}

void Solver::energy(bool with_rate, double out[8]) {
    if (P_.plastic()) throw std::runtime_error("energy diagnostics cover elastic problems only");
    if (with_rate) {
        // dt L(f) at the current state: stage 0 (A = 0 in every RK scheme)
        // with B = 0, so the new fields equal the old ones, slip and state do
        // not move, and the rate register holds dt L(f) (the volume
        // coefficients carry the problem's dt, so the stage uses it too)
        const double b0 = B_[0];
        B_[0] = 0.;
        try {
            if (precision_ == 0)
                stage_impl<double>(dt_, 0, (double)step_index_ * dt_, false);
            else
                stage_impl<float>(dt_, 0, (double)step_index_ * dt_, false);
        } catch (...) {
            B_[0] = b0;
            throw;
        }
        B_[0] = b0;
        cuda_check(cudaGetLastError(), "energy rate stage");
        if (slab_) {
            // the stage wrote only this slab's planes into the other buffer:
            // carry the ghost planes over from the one it read
            const size_t es = precision_ == 0 ? 8 : 4;
            const long long g = ghost_planes();
            for (int side = 0; side < 2; side++) {
                if (side == 0 ? xr0_ == 0 : xr1_ == P_.nx[0]) continue;
                const long long off = (side == 0 ? xr0_ - g : (long long)xr1_) * L_.s0;
                for (int c = 0; c < L_.nfields; c++) {
                    const size_t at = (size_t)(c * L_.cstride + off) * es;
                    cuda_check(cudaMemcpyAsync((char*)F_[cur_] + at, (const char*)F_[1 - cur_] + at,
                                               (size_t)(g * L_.s0) * es, cudaMemcpyDeviceToDevice, stream_),
                               "ghost planes");
                }
            }
        }
    }
    if (!energy_dev_) cuda_check(cudaMalloc(&energy_dev_, 8 * sizeof(double)), "cudaMalloc energy accumulators");
    cuda_check(cudaMemsetAsync(energy_dev_, 0, 8 * sizeof(double), stream_), "memset");
    // geometry in the fields' precision (FP32 problems keep no FP64 copy after set-up)
    if (!J_ || !M_ || !F_[cur_] || !DF_) throw std::runtime_error("energy diagnostics: arrays not allocated");
    for (const auto& B : blocks_) {
        if (precision_ == 0) {
            EnergyArgs<double> a{L_, (const double*)F_[cur_], with_rate ? (const double*)DF_ : nullptr,
                                 (const double*)J_};
            launch_energy<double>(a, B, P_.sbporder, energy_dev_, stream_);
        } else {
            EnergyArgs<float> a{L_, (const float*)F_[cur_], with_rate ? (const float*)DF_ : nullptr,
                                (const float*)J_};
            launch_energy<float>(a, B, P_.sbporder, energy_dev_, stream_);
        }
    }
    for (const auto& I : ifaces_) {
        if (I.kind < 1) continue;
        if (precision_ == 0)
            launch_fault_power<double>(L_, I, blocks_[I.b1], P_.sbporder, (const double*)J_, (const double*)M_,
                                       energy_dev_ + 4, stream_);
        else
            launch_fault_power<float>(L_, I, blocks_[I.b1], P_.sbporder, (const float*)J_, (const float*)M_,
                                      energy_dev_ + 4, stream_);
    }
    cuda_check(cudaGetLastError(), "energy launch");
    fetch_to(energy_dev_, 8 * sizeof(double), out);
    out[2] /= dt_;   // the register holds dt L(f)
    out[3] /= dt_;
}

int Solver::check_status() {
    int st = 0;
    cuda_check(cudaMemcpyAsync(&st, status_, sizeof(int), cudaMemcpyDeviceToHost, stream_), "status");
    cuda_check(cudaMemsetAsync(status_, 0, sizeof(int), stream_), "status reset");
    cuda_check(cudaStreamSynchronize(stream_), "status");
    return st;
}

float Solver::time_steps(int nsteps) {
    cudaEvent_t a, b;
    cuda_check(cudaEventCreate(&a), "event");
    cuda_check(cudaEventCreate(&b), "event");
    cuda_check(cudaEventRecord(a, stream_), "event");
    step(nsteps);
    cuda_check(cudaEventRecord(b, stream_), "event");
    cuda_check(cudaEventSynchronize(b), "event");
    float ms = 0;
    cudaEventElapsedTime(&ms, a, b);
    cudaEventDestroy(a);
    cudaEventDestroy(b);
    return ms;
}

long long Solver::bytes_per_node_stage() const {
    // read and write f and df once each, read the metric and Jacobian once;
    // plastic problems once per step (on the last stage) also read and write
    // the plastic fields and read the heterogeneous initial stress (FP64),
    // counted here per stage, rounded down
    const int esz = precision_ == 0 ? 8 : 4;
    long long b = (long long)(4 * L_.nfields + L_.ndim * L_.ndim + 1) * esz;
    if (P_.plastic()) {
        long long per_step = 2LL * L_.nfieldsp * esz + (S_ ? (long long)L_.ns * 8 : 0);
        b += per_step / std::max(nstages_, 1);
    }
    return b;
}

void Solver::fetch_to(void* devbuf, size_t bytes, void* host) {
    cuda_check(cudaMemcpyAsync(host, devbuf, bytes, cudaMemcpyDeviceToHost, stream_), "d2h");
    cuda_check(cudaStreamSynchronize(stream_), "d2h");
}

void Solver::get_field(int comp, bool absolute, double* out) {
    if (comp < 0 || comp >= L_.nfields + L_.nfieldsp) throw std::runtime_error("field component out of range");
    const size_t n = (size_t)P_.nx[0] * P_.nx[1] * P_.nx[2];
    double* tmp = scratch(n);
    void* base = (comp < L_.nfields) ? F_[cur_] : FP_;
    int c = (comp < L_.nfields) ? comp : comp - L_.nfields;
    if (precision_ == 0)
        launch_fetch_component<double>(L_, (const double*)base, c, absolute && comp < L_.nfields, P_.s0, S_, tmp, stream_);
    else
        launch_fetch_component<float>(L_, (const float*)base, c, absolute && comp < L_.nfields, P_.s0, S_, tmp, stream_);
    fetch_to(tmp, n * sizeof(double), out);
}

void Solver::get_field_noalloc(int comp, bool absolute, double* out) {
    if (comp < 0 || comp >= L_.nfields + L_.nfieldsp) throw std::runtime_error("field component out of range");
    const long long n = (long long)P_.nx[0] * P_.nx[1] * P_.nx[2];
    if (n > FDF_NOALLOC_MAX_VALUES)
        throw std::invalid_argument("field of " + std::to_string(n) + " values exceeds the allocation-free buffer (" +
                                    std::to_string(FDF_NOALLOC_MAX_VALUES) + " values)");
    double* buf = noalloc_field_buffer(device_);
    // the gather kernel writes all n values: nothing has to start at zero
    void* base = (comp < L_.nfields) ? F_[cur_] : FP_;
    int c = (comp < L_.nfields) ? comp : comp - L_.nfields;
    if (precision_ == 0)
        launch_fetch_component<double>(L_, (const double*)base, c, absolute && comp < L_.nfields, P_.s0, S_, buf, stream_);
    else
        launch_fetch_component<float>(L_, (const float*)base, c, absolute && comp < L_.nfields, P_.s0, S_, buf, stream_);
    fetch_to(buf, (size_t)n * sizeof(double), out);
}

void Solver::update_stz_aux() {
    graph_dirty_ = true;
    long long off = 0;
    for (auto& I : ifaces_) {
        if (I.kind != 3) continue;
        I.stz.learned = stz_learned_ ? 1 : 0;
        I.stz.start = stz_start_;
        I.stz.mu_prev = (stz_start_ == 2 && stz_mu_prev_) ? stz_mu_prev_ + off : nullptr;
        off += (long long)I.n0 * I.n1;
        I.stz.mlp = mlp_.ready ? mlp_.dev() : MlpDev{};
        I.stz.stats = stz_counting_ ? stz_counts_ : nullptr;
        I.stz.samples = samples_;
        I.stz.nsamples = nsamples_;
        I.stz.cap = sample_cap_;
    }
}

void Solver::set_stz_start(int mode) {
    if (mode == 1) {
        set_stz_learned(true);
        return;
    }
    if (mode != 0 && mode != 2 && mode != 3) throw std::invalid_argument("STZ start mode must be 0, 1, 2 or 3");
    synchronize();
    stz_learned_ = false;
    stz_start_ = mode;
    if (mode == 2) {   // one slot per node of every STZ interface, none known yet
        long long total = 0;
        for (const auto& I : ifaces_)
            if (I.kind == 3) total += (long long)I.n0 * I.n1;
        if (!stz_mu_prev_ && total > 0)
            cuda_check(cudaMalloc(&stz_mu_prev_, total * sizeof(double)), "cudaMalloc warm-start roots");
        if (stz_mu_prev_) {
            std::vector<double> none((size_t)total, -1.);
            cuda_check(cudaMemcpyAsync(stz_mu_prev_, none.data(), total * sizeof(double), cudaMemcpyHostToDevice,
                                       stream_),
                       "warm-start reset");
            cuda_check(cudaStreamSynchronize(stream_), "warm-start reset");
        }
    }
    update_stz_aux();
}

void Solver::set_stz_learned(bool on) {
    if (on && !mlp_.ready) throw std::invalid_argument("the learned start needs network parameters (init, set or train)");
    synchronize();
    stz_learned_ = on;
    update_stz_aux();
}

void Solver::set_stz_counting(bool on) {
    synchronize();
    if (on && !stz_counts_) {
        cuda_check(cudaMalloc(&stz_counts_, 3 * sizeof(unsigned long long)), "cudaMalloc stz counters");
        cuda_check(cudaMemset(stz_counts_, 0, 3 * sizeof(unsigned long long)), "stz counters");
    }
    stz_counting_ = on;
    update_stz_aux();
}

void Solver::read_stz_counts(long long out[3], bool reset) {
    unsigned long long h[3] = {0, 0, 0};
    if (stz_counts_) {
        cuda_check(cudaMemcpyAsync(h, stz_counts_, sizeof(h), cudaMemcpyDeviceToHost, stream_), "stz counters");
        if (reset) cuda_check(cudaMemsetAsync(stz_counts_, 0, sizeof(h), stream_), "stz counters");
        synchronize();
    }
    for (int i = 0; i < 3; i++) out[i] = (long long)h[i];
}

void Solver::stz_collect(long long capacity) {
    if (capacity < 0) throw std::invalid_argument("negative sample capacity");
    synchronize();
    if (samples_) cudaFree(samples_);
    if (nsamples_) cudaFree(nsamples_);
    samples_ = nullptr;
    nsamples_ = nullptr;
    sample_cap_ = 0;
    if (capacity > 0) {
        cuda_check(cudaMalloc(&samples_, (size_t)capacity * 8 * sizeof(float)), "cudaMalloc samples");
        cuda_check(cudaMalloc(&nsamples_, sizeof(unsigned long long)), "cudaMalloc sample count");
        cuda_check(cudaMemset(nsamples_, 0, sizeof(unsigned long long)), "sample count");
        sample_cap_ = (unsigned long long)capacity;
    }
    update_stz_aux();
}

long long Solver::stz_samples(float* out, long long max) {
    if (!nsamples_) return 0;
    unsigned long long n = 0;
    cuda_check(cudaMemcpyAsync(&n, nsamples_, sizeof(n), cudaMemcpyDeviceToHost, stream_), "sample count");
    synchronize();
    const long long have = (long long)std::min<unsigned long long>(n, sample_cap_);
    const long long k = std::min(have, max);
    if (out && k > 0) {
        cuda_check(cudaMemcpyAsync(out, samples_, (size_t)k * 8 * sizeof(float), cudaMemcpyDeviceToHost, stream_),
                   "samples");
        synchronize();
    }
    return have;
}

void Solver::mlp_train_on_samples(int epochs, int batch, float lr, unsigned long long seed, double* tr,
                                  double* va) {
    const long long have = stz_samples(nullptr, 0);
    mlp_train(mlp_, samples_, have, epochs, batch, lr, seed, tr, va, stream_);
    update_stz_aux();
}

void Solver::set_field(int comp, const double* in) {
    if (comp < 0 || comp >= L_.nfields + L_.nfieldsp) throw std::runtime_error("field component out of range");
    const size_t n = (size_t)P_.nx[0] * P_.nx[1] * P_.nx[2];
    double* tmp = scratch(n);
    cuda_check(cudaMemcpyAsync(tmp, in, n * sizeof(double), cudaMemcpyHostToDevice, stream_), "h2d");
    void* base = (comp < L_.nfields) ? F_[cur_] : FP_;
    int c = (comp < L_.nfields) ? comp : comp - L_.nfields;
    if (precision_ == 0)
        launch_store_component<double>(L_, (double*)base, c, tmp, stream_);
    else
        launch_store_component<float>(L_, (float*)base, c, tmp, stream_);
    synchronize();
}

void Solver::get_rate(int comp, double* out) {
    if (comp < 0 || comp >= L_.nfields) throw std::runtime_error("rate component out of range");
    const size_t n = (size_t)P_.nx[0] * P_.nx[1] * P_.nx[2];
    double* tmp = scratch(n);
    if (precision_ == 0)
        launch_fetch_component<double>(L_, (const double*)DF_, comp, 0, P_.s0, nullptr, tmp, stream_);
    else
        launch_fetch_component<float>(L_, (const float*)DF_, comp, 0, P_.s0, nullptr, tmp, stream_);
    fetch_to(tmp, n * sizeof(double), out);
}

void Solver::set_rate(int comp, const double* in) {
    if (comp < 0 || comp >= L_.nfields) throw std::runtime_error("rate component out of range");
    const size_t n = (size_t)P_.nx[0] * P_.nx[1] * P_.nx[2];
    double* tmp = scratch(n);
    cuda_check(cudaMemcpyAsync(tmp, in, n * sizeof(double), cudaMemcpyHostToDevice, stream_), "h2d");
    if (precision_ == 0)
        launch_store_component<double>(L_, (double*)DF_, comp, tmp, stream_);
    else
        launch_store_component<float>(L_, (float*)DF_, comp, tmp, stream_);
    synchronize();
}

void Solver::get_geometry(int which, int comp, double* out) {
    const size_t n = (size_t)P_.nx[0] * P_.nx[1] * P_.nx[2];
    double* tmp = scratch(n);
    if (which == 0) {
        if (comp < 0 || comp >= L_.ndim) throw std::runtime_error("coordinate component out of range");
        launch_fetch_component<double>(L_, X_, comp, 0, P_.s0, nullptr, tmp, stream_);
    } else if (which == 1 || which == 2) {
        int c = (which == 2) ? 0 : comp;
        if (which == 1 && (comp < 0 || comp >= L_.ndim * L_.ndim)) throw std::runtime_error("metric component out of range");
        const void* base = (which == 2) ? J_ : M_;
        if (precision_ == 0)
            launch_fetch_component<double>(L_, (const double*)base, c, 0, P_.s0, nullptr, tmp, stream_);
        else
            launch_fetch_component<float>(L_, (const float*)base, c, 0, P_.s0, nullptr, tmp, stream_);
    } else {
        throw std::runtime_error("unknown geometry selector");
    }
    fetch_to(tmp, n * sizeof(double), out);
}

static double* fault_array(const IfaceDev& I, int which) {
    switch (which) {
        case 0: return I.u;
        case 1: return I.du;
        case 2: return I.v;
        case 3: return I.s;
        case 4: return I.sn;
        case 5: return I.ux;
        case 6: return I.dux;
        case 7: return I.vx;
        case 8: return I.sx;
        case 9: return I.state;
        case 10: return I.dstate;
        case 11: return I.dstatedt;
        case 12: return I.tfront;
    }
    return nullptr;
}

double* Solver::fault_ptr(int iface, int which) const {
    if (iface < 0 || iface >= (int)ifaces_.size()) return nullptr;
    return fault_array(ifaces_[iface], which);
}

long long Solver::fault_count(int iface, int which) const {
    if (iface < 0 || iface >= (int)ifaces_.size()) return -1;
    const IfaceDev& I = ifaces_[iface];
    if (!fault_array(I, which)) return 0;
    long long nn = (long long)I.n0 * I.n1;
    return (which >= 5 && which <= 8) ? nn * (L_.ndim - 1) : nn;
}

void Solver::get_fault(int iface, int which, double* out) {
    long long n = fault_count(iface, which);
    if (n <= 0) throw std::runtime_error("no such fault array");
    fetch_to(fault_array(ifaces_[iface], which), (size_t)n * sizeof(double), out);
}

cudaEvent_t Solver::ring_event() {
    if (!ring_events_.empty()) {
        cudaEvent_t e = ring_events_.back();
        ring_events_.pop_back();
        return e;
    }
    cudaEvent_t e = nullptr;
    cuda_check(cudaEventCreateWithFlags(&e, cudaEventDisableTiming), "cudaEventCreate");
    return e;
}

void Solver::get_fault_async(int iface, int which, double* out) {
    long long n = fault_count(iface, which);
    if (n <= 0) throw std::runtime_error("no such fault array");
    const size_t bytes = (size_t)n * sizeof(double);
    const double* src = fault_array(ifaces_[iface], which);
    if (capturing_) throw std::runtime_error("get_fault_async inside a capture");
    // ring of snapshots: room for a few steps of every fault array
    const size_t need = (bytes + 255) & ~(size_t)255;
    if (!ring_ || need > ring_cap_ / 4) {
        if (ring_) {   // grow: wait for the copies out of the old ring first
            cuda_check(cudaStreamSynchronize(copy_stream_), "ring");
            for (auto& r : ring_busy_) ring_events_.push_back(r.done);
            ring_busy_.clear();
            cudaFree(ring_);
            ring_ = nullptr;
        }
        size_t cap = (size_t)64 << 20;
        while (cap < 4 * need) cap *= 2;
        cuda_check(cudaMalloc(&ring_, cap), "cudaMalloc read-back ring");
        ring_cap_ = cap;
        ring_head_ = 0;
        if (!copy_stream_)
            cuda_check(cudaStreamCreateWithFlags(&copy_stream_, cudaStreamNonBlocking), "cudaStreamCreate");
    }
    if (ring_head_ + need > ring_cap_) ring_head_ = 0;
    const size_t b0 = ring_head_, b1 = ring_head_ + need;
    // a slot still being copied out: the snapshot waits for that copy (on the device)
    for (size_t q = 0; q < ring_busy_.size();) {
        if (ring_busy_[q].begin < b1 && b0 < ring_busy_[q].end) {
            cuda_check(cudaStreamWaitEvent(stream_, ring_busy_[q].done, 0), "ring wait");
            ring_events_.push_back(ring_busy_[q].done);
            ring_busy_[q] = ring_busy_.back();
            ring_busy_.pop_back();
        } else {
            q++;
        }
    }
    cuda_check(cudaMemcpyAsync(ring_ + b0, src, bytes, cudaMemcpyDeviceToDevice, stream_), "snapshot");
    cudaEvent_t snap = ring_event();
    cuda_check(cudaEventRecord(snap, stream_), "event");
    cuda_check(cudaStreamWaitEvent(copy_stream_, snap, 0), "ring wait");
    ring_events_.push_back(snap);   // reusable once recorded again: waits already captured it
    cuda_check(cudaMemcpyAsync(out, ring_ + b0, bytes, cudaMemcpyDeviceToHost, copy_stream_), "d2h");
    cudaEvent_t done = ring_event();
    cuda_check(cudaEventRecord(done, copy_stream_), "event");
    ring_busy_.push_back({b0, b1, done});
    ring_head_ = b1;
}

void Solver::set_fault(int iface, int which, const double* in) {
    long long n = fault_count(iface, which);
    if (n <= 0) throw std::runtime_error("no such fault array");
    cuda_check(cudaMemcpyAsync(fault_array(ifaces_[iface], which), in, (size_t)n * sizeof(double),
                               cudaMemcpyHostToDevice, stream_),
               "h2d");
    synchronize();
}

}  // namespace fdf
