// Batched ensemble kernels and host driver (compiled with -fmad=false: the
// per-node code is the exact-order volume and interface code, so a member's
// result is bit-identical to the same member run alone in FP32).
//
// One stage of every member is a volume launch per kind of member, then an
// interface launch over all fault tiles.  Members whose 2D blocks all fit the
// tiled 2D kernel (stage_fast2d.cu) are stepped by its batched form, whose
// warps walk a list of (member, block, 32-column tile, row chunk) items --
// bit-identical to the member run alone with that kernel; every other member
// (3D, plastic, small blocks) by the one-thread-per-node kernel below, whose
// CTAs walk the work list of node tiles (grid-stride, one wave of CTAs) --
// bit-identical to the member run alone with the reference-order kernel.  A one-thread
// kernel advances the members' step counters and field-buffer parities at the
// end of each step, so the step sequence holds no host-side state and a chunk
// of steps is captured once in a CUDA graph and replayed.
#include <cuda_runtime.h>

#include <algorithm>
#include <cstddef>
#include <stdexcept>
#include <string>

#include "ensemble.hpp"
#include "iface_dev.cuh"
#include "solver.hpp"
#include "stage_exact.cuh"

namespace fdf {

namespace {

void ck(cudaError_t e, const char* what) {
    if (e != cudaSuccess) throw std::runtime_error(std::string("CUDA error in ") + what + ": " + cudaGetErrorString(e));
}

using RK = EnsRK;

// the per-stage scalars of one member, as the single-problem solver forms them
__device__ __forceinline__ StageArgs member_stage(const EnsMember& M, const RK& rk, int st) {
    StageArgs sa{};
    sa.dt = M.dt;
    sa.A = rk.A[st];
    sa.B = rk.B[st];
    const double t = (double)M.step * M.dt;
    sa.t = t + rk.C[st] * M.dt;
    sa.last = (st + 1 == rk.nstages);
    sa.plastic = 0;
    sa.roundtrip = 0;
    sa.abs_out = 0;
    sa.front_on = M.front_on;
    sa.front_value = M.front_value;
    sa.tfront = (double)(M.step + 1) * M.dt;
    sa.step_dev = nullptr;
    sa.cst = rk.C[st];
    return sa;
}

__global__ void k_ens_volume(const EnsMember* __restrict__ mem, const EnsTile* __restrict__ tiles, int ntiles, RK rk,
                             int st) {
    for (int w = blockIdx.x; w < ntiles; w += gridDim.x) {
        const EnsTile tl = tiles[w];
        const EnsMember& M = mem[tl.m];
        if (M.step >= M.nt) continue;
        const StageArgs sa = member_stage(M, rk, st);
        VolumeArgs<float> va = M.va;
        const int par = M.cur ^ (st & 1);
        va.F = M.buf[par];
        va.Fn = M.buf[par ^ 1];
        const BlockDev& B = M.blk[tl.part];
        for (long long n = tl.begin + threadIdx.x; n < tl.end; n += blockDim.x) {
            if (M.ndim == 3)
                volume_node<float, 3, 2>(va, B, sa, n);
            else if (M.mode == 2)
                volume_node<float, 2, 2>(va, B, sa, n);
            else
                volume_node<float, 2, 3>(va, B, sa, n);
        }
    }
}

__global__ void k_ens_iface(const EnsMember* __restrict__ mem, const EnsTile* __restrict__ tiles, int ntiles, RK rk,
                            int st) {
    for (int w = blockIdx.x; w < ntiles; w += gridDim.x) {
        const EnsTile tl = tiles[w];
        const EnsMember& M = mem[tl.m];
        if (M.step >= M.nt) continue;
        const StageArgs sa = member_stage(M, rk, st);
        IfaceArgs<float> ia = M.ia;
        const int par = M.cur ^ (st & 1);
        ia.F = M.buf[par];
        ia.Fn = M.buf[par ^ 1];
        const IfaceDev& I = M.itf[tl.part];
        for (long long n = tl.begin + threadIdx.x; n < tl.end; n += blockDim.x)
            interface_node<float, false>(ia, I, M.blk[I.b1], M.blk[I.b2], sa, 0, n);
    }
}

__global__ void k_ens_advance(EnsMember* mem, int nmem, int nstages) {
    for (int m = threadIdx.x; m < nmem; m += blockDim.x) {
        if (mem[m].step < mem[m].nt) {
            mem[m].step += 1;
            mem[m].cur ^= (nstages & 1);
        }
    }
}

}  // namespace

Ensemble::Ensemble(const std::vector<std::string>& infiles, int device) : device_(device) {
    if (infiles.empty()) throw std::invalid_argument("empty ensemble");
    ck(cudaSetDevice(device), "cudaSetDevice");
    for (const auto& f : infiles) members_.emplace_back(new Solver(f, 1, device));
    const Solver& s0 = *members_[0];
    nstages_ = s0.nstages_;
    for (int i = 0; i < 5; i++) {
        A_[i] = s0.A_[i];
        B_[i] = s0.B_[i];
    }
    for (int i = 0; i < 6; i++) C_[i] = s0.C_[i];
    std::vector<EnsMember> hm(members_.size());
    for (size_t m = 0; m < members_.size(); m++) {
        Solver& s = *members_[m];
        if (s.nstages_ != nstages_) throw std::invalid_argument("ensemble members must share the Runge-Kutta order");
        if (s.P_.plastic()) throw std::invalid_argument("ensemble members must be elastic");
        if (s.mat_) throw std::invalid_argument("ensemble members must have one material per block");
        if ((int)s.blocks_.size() > ENS_MAX_BLOCKS || s.ifaces_.size() > 2)
            throw std::invalid_argument("ensemble member has too many blocks or interfaces");
        for (const auto& I : s.ifaces_)
            if (I.kind == 3) throw std::invalid_argument("ensemble members use locked, frictionless or slip-weakening interfaces");
        EnsMember& e = hm[m];
        e = EnsMember{};
        VolumeArgs<float>& va = e.va;
        va.L = s.L_;
        va.order = s.P_.sbporder;
        va.cdiss = s.P_.cdiss;
        for (int i = 0; i < 6; i++) va.s0[i] = s.P_.s0[i];
        va.DF = (float*)s.DF_;
        va.M = (const float*)s.M_;
        va.J = (const float*)s.J_;
        va.FP = nullptr;
        va.S = s.S_;
        va.ABS = nullptr;
        va.plastic_tensor = 0;
        IfaceArgs<float>& ia = e.ia;
        ia.L = s.L_;
        for (int i = 0; i < 6; i++) ia.s0[i] = s.P_.s0[i];
        ia.DF = (float*)s.DF_;
        ia.FP = nullptr;
        ia.S = s.S_;
        ia.ABS = nullptr;
        ia.plastic_tensor = 0;
        ia.status = s.status_;
        e.buf[0] = (float*)s.F_[0];
        e.buf[1] = (float*)s.F_[1];
        e.nblocks = (int)s.blocks_.size();
        e.nifaces = (int)s.ifaces_.size();
        for (int b = 0; b < e.nblocks; b++) e.blk[b] = s.blocks_[b];
        for (int i = 0; i < e.nifaces; i++) e.itf[i] = s.ifaces_[i];
        e.ndim = s.L_.ndim;
        e.mode = s.L_.mode;
        e.dt = s.dt_;
        e.nt = s.nt_;
        e.step = s.step_index_;
        e.cur = s.cur_;
        e.front_on = (s.P_.front_on && s.P_.front_field == "V") ? 1 : 0;
        e.front_value = s.P_.front_value;
        host_step_.push_back(e.step);
        host_cur_.push_back(e.cur);
        host_nt_.push_back(e.nt);
    }
    ck(cudaStreamCreateWithFlags(&stream_, cudaStreamNonBlocking), "cudaStreamCreate");
    for (auto& s : members_) s->synchronize();   // set-up done on the members' own streams
    ck(cudaMalloc(&dmem_, hm.size() * sizeof(EnsMember)), "cudaMalloc ensemble table");
    ck(cudaMemcpy(dmem_, hm.data(), hm.size() * sizeof(EnsMember), cudaMemcpyHostToDevice), "ensemble table");
    build_tiles();
}

Ensemble::~Ensemble() {
    if (stream_) cudaStreamSynchronize(stream_);
    if (graph_) cudaGraphExecDestroy(graph_);
    if (dmem_) cudaFree(dmem_);
    if (dvt_) cudaFree(dvt_);
    if (dit_) cudaFree(dit_);
    for (auto& g : g2d_) cudaFree(g.items);
    if (stream_) cudaStreamDestroy(stream_);
}

bool Ensemble::member_tiled2d(int m) const {
    const Solver& s = *members_[m];
    if (s.L_.ndim != 2 || s.P_.cdiss > 0. || s.P_.plastic()) return false;
    for (const auto& B : s.blocks_)
        if (!fast2d_supported(s.L_, B, s.P_.sbporder)) return false;
    return true;
}

void Ensemble::build_tiles() {
    std::vector<EnsTile> vt, it;
    std::vector<std::vector<Ens2dItem>> items2d;
    std::vector<std::pair<int, int>> keys2d;   // (order, mode) of each 2D group
    // rows per tiled-2D work item: `tile` nodes over 32 columns
    const int rows = (int)std::max<long long>(16, cfg_.tile / 32);
    for (size_t m = 0; m < members_.size(); m++) {
        const Solver& s = *members_[m];
        if (member_tiled2d((int)m)) {
            const std::pair<int, int> key(s.P_.sbporder, s.L_.mode);
            size_t g = 0;
            while (g < keys2d.size() && keys2d[g] != key) g++;
            if (g == keys2d.size()) {
                keys2d.push_back(key);
                items2d.emplace_back();
            }
            for (size_t b = 0; b < s.blocks_.size(); b++) {
                const BlockDev& B = s.blocks_[b];
                const int ntj = (B.n[1] + 31) / 32;
                for (int ib = 0; ib < B.n[0]; ib += rows)
                    for (int jt = 0; jt < ntj; jt++)
                        items2d[g].push_back({(int)m, (int)b, jt, ib, std::min(B.n[0], ib + rows)});
            }
        } else {
            for (size_t b = 0; b < s.blocks_.size(); b++) {
                const BlockDev& B = s.blocks_[b];
                const long long nn = (long long)B.n[0] * B.n[1] * B.n[2];
                for (long long a = 0; a < nn; a += cfg_.tile)
                    vt.push_back({(int)m, 0, (int)b, a, std::min(nn, a + cfg_.tile)});
            }
        }
        for (size_t i = 0; i < s.ifaces_.size(); i++) {
            const long long nn = (long long)s.ifaces_[i].n0 * s.ifaces_[i].n1;
            const long long ft = std::max<long long>(cfg_.threads, cfg_.tile / 8);
            for (long long a = 0; a < nn; a += ft) it.push_back({(int)m, 1, (int)i, a, std::min(nn, a + ft)});
        }
    }
    if (dvt_) cudaFree(dvt_);
    if (dit_) cudaFree(dit_);
    dvt_ = dit_ = nullptr;
    for (auto& g : g2d_) cudaFree(g.items);
    g2d_.clear();
    for (size_t g = 0; g < keys2d.size(); g++) {
        Group2d G{keys2d[g].first, keys2d[g].second, 0, (int)items2d[g].size(), nullptr};
        G.grid = fast2d_ensemble_grid(G.order, G.mode, device_);
        ck(cudaMalloc(&G.items, items2d[g].size() * sizeof(Ens2dItem)), "cudaMalloc tiles");
        g2d_.push_back(G);   // owned from here on, freed on rebuild or destruction
        ck(cudaMemcpy(G.items, items2d[g].data(), items2d[g].size() * sizeof(Ens2dItem), cudaMemcpyHostToDevice),
           "tiles");
    }
    nvt_ = (int)vt.size();
    nit_ = (int)it.size();
    ck(cudaMalloc(&dvt_, std::max<size_t>(1, vt.size()) * sizeof(EnsTile)), "cudaMalloc tiles");
    ck(cudaMalloc(&dit_, std::max<size_t>(1, it.size()) * sizeof(EnsTile)), "cudaMalloc tiles");
    if (!vt.empty()) ck(cudaMemcpy(dvt_, vt.data(), vt.size() * sizeof(EnsTile), cudaMemcpyHostToDevice), "tiles");
    if (!it.empty()) ck(cudaMemcpy(dit_, it.data(), it.size() * sizeof(EnsTile), cudaMemcpyHostToDevice), "tiles");
    // one wave of CTAs walks the work lists
    int nsm = 148, occ = 1;
    ck(cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, device_), "device attribute");
    ck(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, k_ens_volume, cfg_.threads, 0), "occupancy");
    grid_ = std::max(1, nsm * std::max(occ, 1));
    if (graph_) {
        cudaGraphExecDestroy(graph_);
        graph_ = nullptr;
    }
}

void Ensemble::set_config(const EnsConfig& c) {
    if (c.threads < 32 || c.threads > 1024 || c.threads % 32 || c.tile < c.threads)
        throw std::invalid_argument("invalid ensemble configuration");
    synchronize();
    cfg_ = c;
    build_tiles();
}

void Ensemble::launch(int nsteps) {
    RK rk{};
    for (int i = 0; i < 5; i++) {
        rk.A[i] = A_[i];
        rk.B[i] = B_[i];
    }
    for (int i = 0; i < 6; i++) rk.C[i] = C_[i];
    rk.nstages = nstages_;
    const int gv = std::min(grid_, std::max(nvt_, 1)), gi = std::min(grid_, std::max(nit_, 1));
    for (int n = 0; n < nsteps; n++) {
        for (int st = 0; st < nstages_; st++) {
            if (nvt_) k_ens_volume<<<gv, cfg_.threads, 0, stream_>>>(dmem_, dvt_, nvt_, rk, st);
            for (const auto& g : g2d_)
                fast2d_ensemble_launch(g.order, g.mode, std::min(g.grid, (g.n + 3) / 4), dmem_, g.items, g.n, rk,
                                       st, stream_);
            if (nit_) k_ens_iface<<<gi, cfg_.threads, 0, stream_>>>(dmem_, dit_, nit_, rk, st);
        }
        k_ens_advance<<<1, 256, 0, stream_>>>(dmem_, (int)members_.size(), nstages_);
    }
    ck(cudaGetLastError(), "ensemble launch");
}

void Ensemble::run(int nsteps) {
    if (nsteps < 0) throw std::invalid_argument("negative step count");
    // work queued on a member's own stream (through its handle) comes first; a
    // member stepped through its handle since the last run: adopt its state
    for (size_t m = 0; m < members_.size(); m++) {
        Solver& s = *members_[m];
        s.synchronize();
        if (s.step_index_ != host_step_[m] || s.cur_ != host_cur_[m]) {
            const int v[2] = {s.step_index_, s.cur_};
            ck(cudaMemcpy(reinterpret_cast<char*>(dmem_ + m) + offsetof(EnsMember, step), v, sizeof(v),
                          cudaMemcpyHostToDevice),
               "ensemble member state");
            host_step_[m] = s.step_index_;
            host_cur_[m] = s.cur_;
        }
    }
    constexpr int CHUNK = 16;
    int left = nsteps;
    if (graph_on_ && left >= CHUNK) {
        if (!graph_) {
            cudaGraph_t g = nullptr;
            ck(cudaStreamBeginCapture(stream_, cudaStreamCaptureModeThreadLocal), "begin capture");
            launch(CHUNK);
            ck(cudaStreamEndCapture(stream_, &g), "end capture");
            ck(cudaGraphInstantiate(&graph_, g, 0), "graph instantiate");
            cudaGraphDestroy(g);
        }
        while (left >= CHUNK) {
            ck(cudaGraphLaunch(graph_, stream_), "graph launch");
            left -= CHUNK;
        }
    }
    if (left > 0) launch(left);
    // the members' own streams (reads through member handles) follow this run
    ck(cudaStreamSynchronize(stream_), "ensemble run");
    for (size_t m = 0; m < members_.size(); m++) {
        const int done = std::min(nsteps, std::max(0, host_nt_[m] - host_step_[m]));
        host_step_[m] += done;
        host_cur_[m] ^= (done * nstages_) & 1;
    }
    sync_members_from_device();
}

void Ensemble::sync_members_from_device() {
    // the members' host-side step index and buffer parity follow the device table
    for (size_t m = 0; m < members_.size(); m++) {
        members_[m]->step_index_ = host_step_[m];
        members_[m]->cur_ = host_cur_[m];
        members_[m]->graph_dirty_ = true;
    }
}

float Ensemble::time_steps(int nsteps) {
    cudaEvent_t e0, e1;
    ck(cudaEventCreate(&e0), "event");
    ck(cudaEventCreate(&e1), "event");
    ck(cudaEventRecord(e0, stream_), "event");
    run(nsteps);
    ck(cudaEventRecord(e1, stream_), "event");
    ck(cudaEventSynchronize(e1), "event");
    float ms = 0.f;
    cudaEventElapsedTime(&ms, e0, e1);
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    return ms;
}

EnsConfig Ensemble::autotune(int steps) {
    if (steps <= 0) throw std::invalid_argument("autotune needs at least one step per candidate");
    const int threads[] = {128, 256};
    const long long tiles[] = {1024, 4096, 16384};
    EnsConfig best = cfg_;
    float best_ms = -1.f;
    const bool g = graph_on_;
    graph_on_ = false;   // candidates are timed on direct launches
    for (int th : threads)
        for (long long tl : tiles) {
            EnsConfig c;
            c.threads = th;
            c.tile = tl;
            set_config(c);
            const float ms = time_steps(steps);
            if (best_ms < 0.f || ms < best_ms) {
                best_ms = ms;
                best = c;
            }
        }
    graph_on_ = g;
    set_config(best);
    return best;
}

long long Ensemble::node_stages_per_step() const {
    long long n = 0;
    for (const auto& s : members_) n += (long long)s->P_.nx[0] * s->P_.nx[1] * s->P_.nx[2];
    return n * nstages_;
}

void Ensemble::synchronize() { ck(cudaStreamSynchronize(stream_), "ensemble synchronize"); }

void Ensemble::check_status() {
    synchronize();
    for (size_t m = 0; m < members_.size(); m++)
        if (int st = members_[m]->check_status())
            throw std::runtime_error("solver status " + std::to_string(st) + " in ensemble member " + std::to_string(m));
}

}  // namespace fdf
