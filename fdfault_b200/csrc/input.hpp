// Host-side description of an fdfault problem, read from the sectioned .in
// text format that fdfault's Python module writes.  The reader keeps the
// reference's semantics: a section starts at the line that equals its header
// exactly, values are read token by token in a fixed order, each reader
// re-opens the file, and the friction/slipweak/stz sections are searched for
// after the interface's own header so several interfaces can share them.
#pragma once

#include "fdf_types.hpp"

#define FDF_MAX_BLOCKS_PER_DIM 16

#include <array>
#include <string>
#include <vector>

namespace fdf {

struct PertSpec {
    int type = 0;   // 0 constant, 1 gaussian, 2 ellipse, 3 linear, 4 boxcar (pert.cpp:54-64)
    double t0 = 0, x0 = 0, dx = 0, y0 = 0, dy = 0;
    double val[9] = {0, 0, 0, 0, 0, 0, 0, 0, 0};
};

struct BlockSpec {
    int coords[3] = {0, 0, 0};
    int nx[3] = {1, 1, 1};
    int xm[3] = {0, 0, 0};
    double rho = 0, lam = 0, g = 0;
    double mu = 0, coh = 0, beta = 0, eta = 0;
    double xb[3] = {0, 0, 0}, lb[3] = {0, 0, 0};
    std::string btype[6];
    std::string bfile[6];
};

struct IfaceSpec {
    std::string kind;
    int direction = 0;
    int idx1[3] = {0, 0, 0}, idx2[3] = {0, 0, 0};
    std::vector<PertSpec> loads;
    std::string loadfile = "none";
    std::vector<PertSpec> perts;
    std::string paramfile = "none";
    double chi0 = 0;
    std::string statefile = "none";
};

struct OutputSpec {
    std::string name, field;
    int tm = 0, tp = 0, ts = 1;
    int xm[3] = {0, 0, 0}, xp[3] = {0, 0, 0}, xs[3] = {1, 1, 1};
};

struct ProblemSpec {
    std::string infile;
    std::string name, datadir;
    int nt = 0;
    double dt = 0, ttot = 0, cfl = 0;
    int ninfo = 1, rkorder = 3;
    int ndim = 3, mode = 2;
    int nx[3] = {1, 1, 1};
    int nblocks[3] = {1, 1, 1};
    std::vector<int> nx_block[3];
    std::vector<int> xm_block[3];
    int sbporder = 4;
    std::string material = "elastic";
    double s0[6] = {0, 0, 0, 0, 0, 0};
    std::string loadfile = "none", matfile = "none";
    bool plastic_tensor = false;
    double cdiss = 0;
    std::vector<BlockSpec> blocks;   // flat index (i*nb1 + j)*nb2 + k
    std::vector<IfaceSpec> ifaces;
    std::vector<OutputSpec> outputs;
    bool front_on = false;
    std::string front_field = "V";
    double front_value = 0;

    bool plastic() const { return material == "plastic"; }
    int nblockstot() const { return nblocks[0] * nblocks[1] * nblocks[2]; }
};

// Reads the whole problem; throws std::runtime_error with the reference's
// message on malformed input.
ProblemSpec read_problem(const std::string& infile);

int pert_type_code(const std::string& s);

}  // namespace fdf
