#pragma once
// Batched ensemble of independent FP32 problems (2D or 3D, elastic) advanced
// together by one persistent cooperative kernel launch per chunk of steps.
//
// Every member is an ordinary Solver (its own fields, geometry, fault arrays,
// status word).  The kernel walks all members in lockstep, stage by stage:
// a grid-stride loop over volume tiles of every active member, a grid-wide
// barrier, a loop over fault tiles, a barrier.  The per-node work is the
// same device code as the per-block kernels (volume_node, interface_node),
// so each member's result is bit-identical to running it alone.  Member step
// counters and field-buffer parities live on the device and are advanced by
// the kernel itself, so the launch can be captured once in a CUDA graph and
// replayed.  Tile size and CTA size come from an autotuner that times each
// candidate on real steps (the tiling does not change any result).
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
    int nstages_ = 0;
    double A_[5] = {0}, B_[5] = {0}, C_[6] = {0};
    bool graph_on_ = true;
    int graph_chunk_ = 0;
    cudaGraphExec_t graph_ = nullptr;
    int grid_ = 0;
    std::vector<int> host_step_, host_cur_, host_nt_;
    void build_tiles();
    void launch(int nsteps);
    void sync_members_from_device();
};

}  // namespace fdf
