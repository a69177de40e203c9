#pragma once
// Batched ensemble of independent FP32 problems (2D or 3D, elastic) advanced
// together, stage by stage, by a few launches per stage.
//
// Every member is an ordinary Solver (its own fields, geometry, fault arrays,
// status word).  Per stage: volume launches whose CTAs (or warps) walk work
// lists covering every active member -- 2D members that fit the tiled 2D
// kernel through its batched form (stage_fast2d.cu), the others through the
// one-thread-per-node kernel -- then one launch over all fault tiles.  The
// per-node work is the same device code as the per-block kernels, so each
// member's result is bit-identical to running it alone with the matching
// kernel.  Member step counters and field-buffer parities live on the device
// and are advanced by a one-thread kernel, so a chunk of steps is captured
// once in a CUDA graph and replayed.  Work-item size and CTA size come from
// an autotuner that times each candidate on real steps (the tiling does not
// change any result).
#include <cuda_runtime.h>

#include <memory>
#include <string>
#include <vector>

#include "fdf_types.hpp"
#include "kernels.hpp"

namespace fdf {

class Solver;

constexpr int ENS_MAX_BLOCKS = 8;

// device table entry of one member
struct EnsMember {
    VolumeArgs<float> va;     // F / Fn chosen per stage from buf[]
    IfaceArgs<float> ia;
    float* buf[2];            // the two field buffers
    BlockDev blk[ENS_MAX_BLOCKS];
    IfaceDev itf[2];
    int nblocks, nifaces, ndim, mode;
    double dt;
    int nt;                   // total steps of the member
    int step;                 // current step index (advanced by the kernel); `cur` follows it
    int cur;                  // buffer read first at the current step
    int front_on;
    double front_value;
};

// a tile: nodes [begin, end) of block (kind 0) or interface (kind 1) `part` of member `m`
struct EnsTile {
    int m, kind, part;
    long long begin, end;
};

// a work item of the tiled 2D volume kernel: 32-column tile jt of block
// `part` of member `m`, rows [ib, ie)
struct Ens2dItem {
    int m, part, jt, ib, ie;
};

// Runge-Kutta coefficients shared by all members
struct EnsRK {
    double A[5], B[5], C[6];
    int nstages;
};

// tiled 2D volume stage over a work list (stage_fast2d.cu)
int fast2d_ensemble_grid(int order, int mode, int device);
void fast2d_ensemble_launch(int order, int mode, int grid, const EnsMember* mem, const Ens2dItem* items,
                            int nitems, const EnsRK& rk, int st, cudaStream_t s);

struct EnsConfig {
    int threads = 256;        // CTA size
    long long tile = 4096;    // nodes per tile
};

class Ensemble {
  public:
    Ensemble(const std::vector<std::string>& infiles, int device);
    ~Ensemble();
    int size() const { return (int)members_.size(); }
    Solver& member(int i) { return *members_.at(i); }
    // advance every member by min(nsteps, its remaining steps)
    void run(int nsteps);
    float time_steps(int nsteps);   // device time of run(nsteps), ms (CUDA events)
    // time `steps` steps with each candidate configuration (real steps: the
    // members advance) and keep the fastest; returns the chosen config
    EnsConfig autotune(int steps);
    void set_config(const EnsConfig& c);
    EnsConfig config() const { return cfg_; }
    void use_graph(bool on) { graph_on_ = on; }
    long long node_stages_per_step() const;   // sum over active members
    int device() const { return device_; }
    void synchronize();
    void check_status();

  private:
    std::vector<std::unique_ptr<Solver>> members_;
    int device_ = 0;
    cudaStream_t stream_ = nullptr;
    EnsConfig cfg_;
    EnsMember* dmem_ = nullptr;
    EnsTile* dvt_ = nullptr;
    EnsTile* dit_ = nullptr;
    int nvt_ = 0, nit_ = 0;
    // tiled 2D work lists, one per (order, mode) group of members
    struct Group2d {
        int order, mode, grid, n;
        Ens2dItem* items;
    };
    std::vector<Group2d> g2d_;
    int nstages_ = 0;
    double A_[5] = {0}, B_[5] = {0}, C_[6] = {0};
    bool graph_on_ = true;
    int graph_chunk_ = 0;
    cudaGraphExec_t graph_ = nullptr;
    int grid_ = 0;
    std::vector<int> host_step_, host_cur_, host_nt_;
    void build_tiles();
    bool member_tiled2d(int m) const;   // stepped by the tiled 2D kernel
    void launch(int nsteps);
    void sync_members_from_device();
};

}  // namespace fdf
