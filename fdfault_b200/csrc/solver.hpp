// Host orchestration of one fdfault problem on one GPU.
//
// Construction mirrors problem::problem + domain::domain (src/problem.cpp:16-84,
// src/domain.cpp:19-153): read the .in file, build the grid and metrics on the
// device, boundary and interface normals, friction parameters, the time step,
// the initial interface solve, the initial absolute-stress round trip and the
// initial front.  do_rk_stage() is the drop-in for domain::do_rk_stage
// (src/domain.cpp:228-305) and step() for one pass of the loop body of
// problem::solve (src/problem.cpp:151-168).
#pragma once

#include <cuda_runtime.h>

#include <memory>
#include <string>
#include <vector>

#include "fdf_types.hpp"
#include "input.hpp"
#include "kernels.hpp"
#include "mlp.hpp"

namespace fdf {

class OutputList;

class Solver {
  public:
    Solver(const std::string& infile, int precision, int device);
    ~Solver();
    Solver(const Solver&) = delete;
    Solver& operator=(const Solver&) = delete;

    // one Runge-Kutta stage of one time step (domain::do_rk_stage)
    void do_rk_stage(double dt, int stage, double t);
    // nsteps full steps starting at the current step counter
    void step(int nsteps);
    // the whole problem::solve loop including output units and fronts
    void solve();
    // stage `stage` of the current step exactly as step() runs it; the last
    // stage advances the step counter (stages must come in order)
    void step_stage(int stage);

    // x slabs (fields.cpp:276-291, cartesian.cpp:88-165 split the domain the
    // same way across MPI ranks): this process updates the global x planes
    // [x0, x1) and reads order-1 ghost planes on each side, which the caller
    // refreshes after every stage from the neighbouring slabs (pack_ghosts /
    // unpack_ghosts).  (0, nx) is the whole domain.
    void set_x_range(int x0, int x1);
    bool slab() const { return slab_; }
    int ghost_planes() const { return P_.sbporder - 1; }
    long long ghost_count() const;   // elements of one side's ghost exchange
    // side 0: the first ghost_planes() updated planes (the lower neighbour's
    // upper ghosts); side 1: the last ones.  dst/src are device buffers of
    // ghost_count() elements in the fields' precision.
    void pack_ghosts(int side, void* dst);
    // side 0: the ghost planes below x0; side 1: those from x1 on
    void unpack_ghosts(int side, const void* src);
    // run on the caller's stream (own = false) or the handle's own (own = true)
    void set_stream(bool own, cudaStream_t s);

    // reset the step counter (tests that drive stages directly)
    void set_step_index(int i) { step_index_ = i; }
    int step_index() const { return step_index_; }

    // host <-> device access in the reference's unpadded node order
    void get_field(int comp, bool absolute, double* out);
    // same values as get_field, gathered into the fixed static device buffer
    // (noalloc.hpp) instead of the growable scratch buffer; never allocates
    void get_field_noalloc(int comp, bool absolute, double* out);
    void set_field(int comp, const double* in);
    void get_rate(int comp, double* out);
    void set_rate(int comp, const double* in);
    void get_geometry(int which, int comp, double* out);
    // volume component as the output list writes it at step tstep (absolute stress)
    void fetch_output_component(int comp, int tstep, double* out);
    void get_fault(int iface, int which, double* out);
    void get_fault_async(int iface, int which, double* out);   // queued on the stream, no wait
    double* fault_ptr(int iface, int which) const;   // device array of a fault quantity (or null)
    void set_fault(int iface, int which, const double* in);
    long long fault_count(int iface, int which) const;

    // STZ friction: learned Newton start, counters, solver-generated samples
    void set_stz_learned(bool on);
    // start of the plain STZ Newton solve: 0 bracket midpoint (reference), 2
    // warm start from each node's previous root, 3 midpoint with the exact
    // derivative (1 is the learned start, set_stz_learned)
    void set_stz_start(int mode);
    void set_plastic_rule(int rule);
    int plastic_rule() const { return plastic_rule_; }
    void set_stz_counting(bool on);
    void read_stz_counts(long long out[3], bool reset);
    void stz_collect(long long capacity);            // 0 stops collecting and frees the buffer
    long long stz_samples(float* out, long long max);  // copies min(count, max) rows of 8 floats
    MlpState& mlp() { return mlp_; }
    void refresh_stz() { synchronize(); update_stz_aux(); }   // after the network's buffers change
    void mlp_train_on_samples(int epochs, int batch, float lr, unsigned long long seed, double* tr, double* va);

    // FP64 energy diagnostics (elastic problems): out[0] kinetic, out[1] strain
    // energy, out[2] their rate under the semi-discrete operator at the current
    // state (with_rate; computed by a stage evaluation that leaves fields, slip
    // and state unchanged and dt L(f) in the rate register), out[3] the
    // sum of the rate terms' magnitudes, out[4] the frictional power of all
    // interfaces, out[5..7] zero
    void energy(bool with_rate, double out[8]);
    void synchronize();
    int check_status();            // reads and clears the device status word
    float time_steps(int nsteps);  // device time of nsteps steps, ms (CUDA events on the solver stream)
    void set_profile(bool on);
    void profile_read(int kernel, double* total_ms, long long* launches);
    void use_fast_kernel(bool on) { set_volume_kernel(on ? 1 : 0); }
    // FP32 3D volume kernel: 0 one thread per node (reference order), 1 tiled
    // (per-thread global loads), 2 staged (bulk copies into shared memory),
    // 3 register window (x window in registers, tile planes staged by TMA)
    void set_volume_kernel(int kind) {
        vkernel_ = kind;
        graph_dirty_ = true;
    }
    int volume_kernel_active() const;   // the kind that runs (0 when the chosen one does not apply)
    // polls of a bounded wait for staged data (<= 0: the built-in limit)
    void set_wait_limit(long long polls) {
        wait_limit_ = polls != 0 ? polls : (1LL << 22);
        graph_dirty_ = true;
    }
    // replay steps from a captured CUDA graph of two steps (default on)
    void use_graphs(bool on) { graphs_ = on; }
    bool graphs() const { return graphs_; }
    bool fast_kernel_active() const;

    const ProblemSpec& spec() const { return P_; }
    const Layout& layout() const { return L_; }
    int precision() const { return precision_; }
    int device() const { return device_; }
    double dt() const { return dt_; }
    int nt() const { return nt_; }
    int nstages() const { return nstages_; }
    double ttot() const { return ttot_; }
    double cfl() const { return cfl_; }
    cudaStream_t stream() const { return stream_; }
    const std::vector<IfaceDev>& ifaces() const { return ifaces_; }
    const std::vector<BlockDev>& blocks() const { return blocks_; }
    long long bytes_per_node_stage() const;

    // raw device pointers (for output units and tests)
    void* field_ptr() const { return F_[cur_]; }
    const double* x_ptr() const { return X_; }

  private:
    friend class OutputList;
    friend class Ensemble;
    template <typename T>
    void stage_impl(double dt, int stage, double t, bool for_step);
    template <typename T>
    void init_fields();
    void setup_geometry();
    std::vector<double> setup_material();
    void setup_plastic_visits(const std::vector<double>& mat);
    void apply_plastic_rule();
    void check_plastic_rule() const;
    void setup_boundaries();
    void setup_interfaces();
    void set_time_step();
    void set_block_coefficients();
    void initial_interface_solve();
    void launch_volume(int b, const StageArgs& sa);
    void fetch_to(void* devbuf, size_t bytes, void* host);
    double* scratch(size_t n);

    ProblemSpec P_;
    Layout L_{};
    int precision_ = 0;   // 0 exact FP64, 1 FP32 fields
    int device_ = 0;
    cudaStream_t stream_ = nullptr;
    cudaStream_t own_stream_ = nullptr;   // created by the handle; stream_ may be the caller's
    // get_fault_async: the array is snapshotted on stream_ into a device ring
    // and copied to the host on copy_stream_, overlapping the steps queued after
    struct RingCopy {
        size_t begin, end;
        cudaEvent_t done;   // the host copy out of [begin, end) finished
    };
    cudaStream_t copy_stream_ = nullptr;
    char* ring_ = nullptr;
    size_t ring_cap_ = 0, ring_head_ = 0;
    std::vector<RingCopy> ring_busy_;
    std::vector<cudaEvent_t> ring_events_;   // free events (timing disabled)
    cudaEvent_t ring_event();
    bool slab_ = false;                   // x range narrower than the domain
    int xr0_ = 0, xr1_ = 0;               // updated global x planes [xr0_, xr1_)
    int stage_next_ = 0;                  // next stage of step_stage
    double dt_ = 0, ttot_ = 0, cfl_ = 0;
    int nt_ = 0, nstages_ = 0;
    double A_[5] = {0}, B_[5] = {0}, C_[6] = {0};
    int step_index_ = 0;
    int vkernel_ = 3;   // FP32 default: register-window 3D kernel (2D: the tiled 2D kernel)
    StagedMapsHost* staged_maps_ = nullptr;   // tensor maps of the FP32 arrays (staged kernel)
    RegMapsHost* reg_maps_ = nullptr;         // tensor maps of the FP32 arrays (register-window kernel)
    long long wait_limit_ = 1LL << 22;        // polls of a bounded mbarrier wait (TMA-staged kernels)
    double* energy_dev_ = nullptr;            // 8 FP64 accumulators of the energy diagnostics

    // device buffers
    void* F_[2] = {nullptr, nullptr};
    int cur_ = 0;
    void* DF_ = nullptr;
    void* FP_ = nullptr;
    void* M_ = nullptr;
    void* J_ = nullptr;
    double* M64_ = nullptr;
    double* J64_ = nullptr;
    double* X_ = nullptr;
    double* S_ = nullptr;
    double* mat_ = nullptr;   // heterogeneous material planes rho, lambda, G (FP64) or null
    // plastic return map: 0 the reference's loop (truncated modulus, the nodes
    // its z loop reaches), 1 every node with the exact modulus
    int plastic_rule_ = 0;
    int pvisit_ref_ = 0;                  // pvisit of the reference rule (0, 1 or 2)
    unsigned char* pmask_ = nullptr;      // nodes the reference's z loop reaches (pvisit 2)
    std::string plastic_stuck_;           // why the reference's loop would not finish, or empty
    double* ABS_ = nullptr;
    int* status_ = nullptr;
    double* scratch_ = nullptr;
    size_t scratch_n_ = 0;
    std::vector<void*> owned_;   // face normals, fault arrays, parameter shapes

    std::vector<BlockDev> blocks_;
    BlockDev* blocks_dev_ = nullptr;   // device copy of blocks_ (final after set-up)
    std::vector<IfaceDev> ifaces_;
    MlpState mlp_;
    bool stz_learned_ = false;
    int stz_start_ = 0;
    double* stz_mu_prev_ = nullptr;   // per interface node of all STZ interfaces (warm start)
    unsigned long long* stz_counts_ = nullptr;   // device [3]
    bool stz_counting_ = false;
    float* samples_ = nullptr;                   // device [cap][8]
    unsigned long long* nsamples_ = nullptr;
    unsigned long long sample_cap_ = 0;
    void update_stz_aux();
    // CUDA graph of two steps, replayed by step() when no output is due
    bool graphs_ = true;
    bool graph_dirty_ = true;
    bool capturing_ = false;
    int* step_dev_ = nullptr;
    cudaGraphExec_t graph_exec_[2] = {nullptr, nullptr};   // one per field-buffer parity
    void step_launches(int nsteps);
    void step_graph(int nsteps);
    std::unique_ptr<OutputList> out_;

    // profiling
    bool profile_ = false;
    std::vector<cudaEvent_t> ev_pool_;
    std::vector<std::pair<int, std::pair<cudaEvent_t, cudaEvent_t>>> ev_pending_;
    double prof_ms_[4] = {0, 0, 0, 0};
    long long prof_n_[4] = {0, 0, 0, 0};
    void prof_flush();
    cudaEvent_t ev_get();
    void* dalloc(size_t bytes);
};

void cuda_check(cudaError_t e, const char* what);

}  // namespace fdf
