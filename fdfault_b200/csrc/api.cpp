// C ABI (include/fdfault_b200.h) over the Solver class.  No C++ exception
// crosses this boundary: every entry point converts failures into a negative
// status and keeps the message for fdf_last_error().
#include "../../include/fdfault_b200.h"

#include <cuda_runtime.h>

#include <cstring>
#include <stdexcept>
#include <string>

#include "ensemble.hpp"
#include "solver.hpp"

struct fdf_handle {
    fdf::Solver* s = nullptr;
    std::string err;
    bool borrowed = false;   // a member of an ensemble: the ensemble owns the solver
};

struct fdf_ensemble {
    fdf::Ensemble* e = nullptr;
    std::string err;
};

namespace {

thread_local std::string g_create_error;

// Makes a handle's device current for the duration of one call and restores
// the caller's device afterwards, so one host thread may drive handles on
// several devices: every allocation, launch and per-device lookup of a call
// then happens on the handle's own device.
class DeviceGuard {
  public:
    explicit DeviceGuard(int device) {
        if (cudaGetDevice(&prev_) != cudaSuccess) prev_ = -1;
        if (prev_ != device) {
            if (cudaSetDevice(device) != cudaSuccess)
                throw std::runtime_error("CUDA error in cudaSetDevice for the handle's device");
            changed_ = true;
        }
    }
    ~DeviceGuard() {
        if (changed_ && prev_ >= 0) cudaSetDevice(prev_);
    }
    DeviceGuard(const DeviceGuard&) = delete;
    DeviceGuard& operator=(const DeviceGuard&) = delete;

  private:
    int prev_ = -1;
    bool changed_ = false;
};

// Restores the caller's current device on exit (construction sets the new
// handle's device itself, after the input has been read and checked).
class DeviceRestore {
  public:
    DeviceRestore() {
        if (cudaGetDevice(&prev_) != cudaSuccess) prev_ = -1;
    }
    ~DeviceRestore() {
        int now = -1;
        if (prev_ >= 0 && cudaGetDevice(&now) == cudaSuccess && now != prev_) cudaSetDevice(prev_);
    }
    DeviceRestore(const DeviceRestore&) = delete;
    DeviceRestore& operator=(const DeviceRestore&) = delete;

  private:
    int prev_ = -1;
};

template <typename F>
int guarded(fdf_handle* h, F&& f) {
    if (!h || !h->s) return FDF_ERR_ARG;
    try {
        DeviceGuard dg(h->s->device());
        f(*h->s);
        return 0;
    } catch (const std::exception& e) {
        h->err = e.what();
        if (h->err.find("solver status") != std::string::npos) return FDF_ERR_SOLVER;
        if (h->err.find("cuda") != std::string::npos || h->err.find("CUDA") != std::string::npos) return FDF_ERR_CUDA;
        return FDF_ERR_ARG;
    }
}

template <typename F>
int eguarded(fdf_ensemble* h, F&& f) {
    if (!h || !h->e) return FDF_ERR_ARG;
    try {
        DeviceGuard dg(h->e->device());
        f(*h->e);
        return 0;
    } catch (const std::exception& e) {
        h->err = e.what();
        if (h->err.find("solver status") != std::string::npos) return FDF_ERR_SOLVER;
        if (h->err.find("CUDA") != std::string::npos || h->err.find("cuda") != std::string::npos) return FDF_ERR_CUDA;
        return FDF_ERR_ARG;
    }
}


}  // namespace

extern "C" {

int fdf_create(const char* infile, int precision, int device, fdf_handle** out) {
    if (!infile || !out) return FDF_ERR_ARG;
    *out = nullptr;
    try {
        fdf_handle* h = new fdf_handle;
        try {
            DeviceRestore dr;   // the caller's current device is restored on return
            h->s = new fdf::Solver(infile, precision, device);
        } catch (...) {
            delete h;
            throw;
        }
        *out = h;
        return 0;
    } catch (const std::exception& e) {
        g_create_error = e.what();
        std::string m = g_create_error;
        if (m.find("cuda") != std::string::npos) return FDF_ERR_CUDA;
        return FDF_ERR_INPUT;
    }
}

void fdf_destroy(fdf_handle* h) {
    if (!h) return;
    try {
        if (!h->borrowed && h->s) {
            DeviceGuard dg(h->s->device());
            delete h->s;
        }
    } catch (...) {
    }
    delete h;
}

int fdf_get_info(fdf_handle* h, int* ints, double* dbls) {
    if (!ints || !dbls) return FDF_ERR_ARG;
    return guarded(h, [&](fdf::Solver& s) {
        const auto& P = s.spec();
        const auto& L = s.layout();
        ints[0] = P.ndim;
        ints[1] = P.mode;
        ints[2] = P.nx[0];
        ints[3] = P.nx[1];
        ints[4] = P.nx[2];
        ints[5] = L.nfields;
        ints[6] = L.nfieldsp;
        ints[7] = (int)P.ifaces.size();
        ints[8] = s.nstages();
        ints[9] = s.nt();
        ints[10] = P.sbporder;
        ints[11] = P.nblocks[0];
        ints[12] = P.nblocks[1];
        ints[13] = P.nblocks[2];
        ints[14] = P.plastic() ? 1 : 0;
        ints[15] = P.rkorder;
        dbls[0] = s.dt();
        dbls[1] = s.ttot();
        dbls[2] = s.cfl();
    });
}

int fdf_do_rk_stage(fdf_handle* h, double dt, int stage, double t) {
    return guarded(h, [&](fdf::Solver& s) { s.do_rk_stage(dt, stage, t); });
}

int fdf_step(fdf_handle* h, int nsteps) {
    if (nsteps < 0) return FDF_ERR_ARG;
    return guarded(h, [&](fdf::Solver& s) { s.step(nsteps); });
}

int fdf_solve(fdf_handle* h) {
    return guarded(h, [&](fdf::Solver& s) { s.solve(); });
}

int fdf_step_stage(fdf_handle* h, int stage) {
    return guarded(h, [&](fdf::Solver& s) { s.step_stage(stage); });
}

int fdf_set_x_range(fdf_handle* h, int x0, int x1) {
    return guarded(h, [&](fdf::Solver& s) { s.set_x_range(x0, x1); });
}

int fdf_ghost_info(fdf_handle* h, int* planes, long long* count, int* elem_bytes) {
    if (!planes || !count || !elem_bytes) return FDF_ERR_ARG;
    return guarded(h, [&](fdf::Solver& s) {
        *planes = s.ghost_planes();
        *count = s.ghost_count();
        *elem_bytes = s.precision() == 0 ? 8 : 4;
    });
}

int fdf_pack_ghosts(fdf_handle* h, int side, void* dst) {
    if (!dst) return FDF_ERR_ARG;
    return guarded(h, [&](fdf::Solver& s) { s.pack_ghosts(side, dst); });
}

int fdf_unpack_ghosts(fdf_handle* h, int side, const void* src) {
    if (!src) return FDF_ERR_ARG;
    return guarded(h, [&](fdf::Solver& s) { s.unpack_ghosts(side, src); });
}

int fdf_get_block(fdf_handle* h, int block, int* lo, int* n) {
    if (!lo || !n) return FDF_ERR_ARG;
    return guarded(h, [&](fdf::Solver& s) {
        if (block < 0 || block >= (int)s.blocks().size()) throw std::runtime_error("block index out of range");
        for (int d = 0; d < 3; d++) {
            lo[d] = s.blocks()[block].lo[d];
            n[d] = s.blocks()[block].n[d];
        }
    });
}

int fdf_get_interface(fdf_handle* h, int iface, int* direction, int* lo, int* n) {
    if (!direction || !lo || !n) return FDF_ERR_ARG;
    return guarded(h, [&](fdf::Solver& s) {
        if (iface < 0 || iface >= (int)s.ifaces().size()) throw std::runtime_error("interface index out of range");
        const fdf::IfaceDev& I = s.ifaces()[iface];
        *direction = I.direction;
        for (int d = 0; d < 3; d++) lo[d] = I.mlb[d];
        n[0] = I.n0;
        n[1] = I.n1;
    });
}

int fdf_set_stream(fdf_handle* h, int own, void* stream) {
    return guarded(h, [&](fdf::Solver& s) { s.set_stream(own != 0, static_cast<cudaStream_t>(stream)); });
}

int fdf_get_step(fdf_handle* h, int* step) {
    if (!step) return FDF_ERR_ARG;
    return guarded(h, [&](fdf::Solver& s) { *step = s.step_index(); });
}

int fdf_set_step(fdf_handle* h, int step) {
    if (step < 0) return FDF_ERR_ARG;
    return guarded(h, [&](fdf::Solver& s) { s.set_step_index(step); });
}

int fdf_get_field(fdf_handle* h, int comp, int absolute, double* out) {
    if (!out) return FDF_ERR_ARG;
    return guarded(h, [&](fdf::Solver& s) { s.get_field(comp, absolute != 0, out); });
}

int fdf_get_field_noalloc(fdf_handle* h, int comp, int absolute, double* out) {
    if (!out) return FDF_ERR_ARG;
    return guarded(h, [&](fdf::Solver& s) { s.get_field_noalloc(comp, absolute != 0, out); });
}

int fdf_set_field(fdf_handle* h, int comp, const double* in) {
    if (!in) return FDF_ERR_ARG;
    return guarded(h, [&](fdf::Solver& s) { s.set_field(comp, in); });
}

int fdf_get_rate(fdf_handle* h, int comp, double* out) {
    if (!out) return FDF_ERR_ARG;
    return guarded(h, [&](fdf::Solver& s) { s.get_rate(comp, out); });
}

int fdf_set_rate(fdf_handle* h, int comp, const double* in) {
    if (!in) return FDF_ERR_ARG;
    return guarded(h, [&](fdf::Solver& s) { s.set_rate(comp, in); });
}

int fdf_get_geometry(fdf_handle* h, int which, int comp, double* out) {
    if (!out) return FDF_ERR_ARG;
    return guarded(h, [&](fdf::Solver& s) { s.get_geometry(which, comp, out); });
}

int fdf_fault_count(fdf_handle* h, int iface, int which, long long* n) {
    if (!n) return FDF_ERR_ARG;
    return guarded(h, [&](fdf::Solver& s) {
        long long c = s.fault_count(iface, which);
        if (c < 0) throw std::runtime_error("interface index out of range");
        *n = c;
    });
}

int fdf_get_fault(fdf_handle* h, int iface, int which, double* out) {
    if (!out) return FDF_ERR_ARG;
    return guarded(h, [&](fdf::Solver& s) { s.get_fault(iface, which, out); });
}

int fdf_get_fault_async(fdf_handle* h, int iface, int which, double* out) {
    if (!out) return FDF_ERR_ARG;
    return guarded(h, [&](fdf::Solver& s) { s.get_fault_async(iface, which, out); });
}

int fdf_set_fault(fdf_handle* h, int iface, int which, const double* in) {
    if (!in) return FDF_ERR_ARG;
    return guarded(h, [&](fdf::Solver& s) { s.set_fault(iface, which, in); });
}

int fdf_synchronize(fdf_handle* h) {
    return guarded(h, [&](fdf::Solver& s) {
        s.synchronize();
        if (int st = s.check_status()) throw std::runtime_error("solver status " + std::to_string(st));
    });
}

int fdf_time_steps(fdf_handle* h, int nsteps, double* ms) {
    if (!ms || nsteps < 0) return FDF_ERR_ARG;
    return guarded(h, [&](fdf::Solver& s) { *ms = (double)s.time_steps(nsteps); });
}

int fdf_profile(fdf_handle* h, int on) {
    return guarded(h, [&](fdf::Solver& s) { s.set_profile(on != 0); });
}

int fdf_profile_read(fdf_handle* h, int kernel, double* total_ms, long long* launches) {
    if (!total_ms || !launches) return FDF_ERR_ARG;
    return guarded(h, [&](fdf::Solver& s) { s.profile_read(kernel, total_ms, launches); });
}

int fdf_use_graphs(fdf_handle* h, int on) {
    return guarded(h, [&](fdf::Solver& s) { s.use_graphs(on != 0); });
}

int fdf_set_volume_kernel(fdf_handle* h, int kind, int* active) {
    if (kind < 0 || kind > 3) return FDF_ERR_ARG;
    return guarded(h, [&](fdf::Solver& s) {
        s.set_volume_kernel(kind);
        if (active) *active = s.volume_kernel_active();
    });
}

int fdf_energy(fdf_handle* h, int with_rate, double out[8]) {
    if (!out) return FDF_ERR_ARG;
    return guarded(h, [&](fdf::Solver& s) { s.energy(with_rate != 0, out); });
}

int fdf_set_wait_limit(fdf_handle* h, long long polls) {
    return guarded(h, [&](fdf::Solver& s) { s.set_wait_limit(polls); });
}

int fdf_use_fast_kernel(fdf_handle* h, int on, int* active) {
    return guarded(h, [&](fdf::Solver& s) {
        s.use_fast_kernel(on != 0);
        if (active) *active = s.fast_kernel_active() ? 1 : 0;
    });
}

int fdf_bytes_per_node_stage(fdf_handle* h, long long* bytes) {
    if (!bytes) return FDF_ERR_ARG;
    return guarded(h, [&](fdf::Solver& s) { *bytes = s.bytes_per_node_stage(); });
}

int fdf_set_plastic_rule(fdf_handle* h, int rule) {
    return guarded(h, [&](fdf::Solver& s) { s.set_plastic_rule(rule); });
}

int fdf_stz_set_start(fdf_handle* h, int mode) {
    return guarded(h, [&](fdf::Solver& s) { s.set_stz_start(mode); });
}

int fdf_stz_set_learned(fdf_handle* h, int on) {
    return guarded(h, [&](fdf::Solver& s) { s.set_stz_learned(on != 0); });
}

int fdf_stz_set_counting(fdf_handle* h, int on) {
    return guarded(h, [&](fdf::Solver& s) { s.set_stz_counting(on != 0); });
}

int fdf_stz_read_counts(fdf_handle* h, long long* counts, int reset) {
    if (!counts) return FDF_ERR_ARG;
    return guarded(h, [&](fdf::Solver& s) { s.read_stz_counts(counts, reset != 0); });
}

int fdf_stz_collect(fdf_handle* h, long long capacity) {
    return guarded(h, [&](fdf::Solver& s) { s.stz_collect(capacity); });
}

int fdf_stz_samples(fdf_handle* h, float* out, long long max_rows, long long* count) {
    if (!count || max_rows < 0 || (max_rows > 0 && !out)) return FDF_ERR_ARG;
    return guarded(h, [&](fdf::Solver& s) { *count = s.stz_samples(out, max_rows); });
}

int fdf_mlp_init(fdf_handle* h, unsigned long long seed) {
    return guarded(h, [&](fdf::Solver& s) {
        s.synchronize();
        fdf::mlp_init(s.mlp(), seed, s.stream());
        s.refresh_stz();
    });
}

int fdf_mlp_set_params(fdf_handle* h, const float* params) {
    if (!params) return FDF_ERR_ARG;
    return guarded(h, [&](fdf::Solver& s) {
        s.synchronize();
        fdf::mlp_set_params(s.mlp(), params, s.stream());
        s.refresh_stz();
    });
}

int fdf_mlp_get_params(fdf_handle* h, float* params) {
    if (!params) return FDF_ERR_ARG;
    return guarded(h, [&](fdf::Solver& s) { fdf::mlp_get_params(s.mlp(), params, s.stream()); });
}

int fdf_mlp_infer(fdf_handle* h, const float* x, long long n, float* y, int force_thread) {
    if (n < 0 || (n > 0 && (!x || !y))) return FDF_ERR_ARG;
    return guarded(h, [&](fdf::Solver& s) { fdf::mlp_infer(s.mlp(), x, n, y, force_thread, s.stream()); });
}

int fdf_mlp_gradients(fdf_handle* h, const float* x, const float* t, long long n, float* grads, double* loss) {
    if (!x || !t || !grads || !loss || n <= 0) return FDF_ERR_ARG;
    return guarded(h, [&](fdf::Solver& s) { fdf::mlp_gradients(s.mlp(), x, t, n, grads, loss, s.stream()); });
}

int fdf_mlp_train(fdf_handle* h, int epochs, int batch, float lr, unsigned long long seed, double* train_loss,
                  double* val_loss) {
    if (!train_loss || !val_loss) return FDF_ERR_ARG;
    return guarded(h, [&](fdf::Solver& s) {
        s.synchronize();
        s.mlp_train_on_samples(epochs, batch, lr, seed, train_loss, val_loss);
        s.refresh_stz();
    });
}

int fdf_ensemble_create(const char* const* infiles, int n, int device, fdf_ensemble** out) {
    if (!infiles || n <= 0 || !out) return FDF_ERR_ARG;
    *out = nullptr;
    try {
        std::vector<std::string> files;
        for (int i = 0; i < n; i++) {
            if (!infiles[i]) return FDF_ERR_ARG;
            files.emplace_back(infiles[i]);
        }
        fdf_ensemble* h = new fdf_ensemble;
        try {
            DeviceRestore dr;   // the caller's current device is restored on return
            h->e = new fdf::Ensemble(files, device);
        } catch (...) {
            delete h;
            throw;
        }
        *out = h;
        return 0;
    } catch (const std::exception& e) {
        g_create_error = e.what();
        std::string m = g_create_error;
        if (m.find("CUDA") != std::string::npos || m.find("cuda") != std::string::npos) return FDF_ERR_CUDA;
        return FDF_ERR_INPUT;
    }
}

void fdf_ensemble_destroy(fdf_ensemble* h) {
    if (!h) return;
    try {
        if (h->e) {
            DeviceGuard dg(h->e->device());
            delete h->e;
        }
    } catch (...) {
    }
    delete h;
}

int fdf_ensemble_size(fdf_ensemble* h, int* n) {
    if (!n) return FDF_ERR_ARG;
    return eguarded(h, [&](fdf::Ensemble& e) { *n = e.size(); });
}

int fdf_ensemble_member(fdf_ensemble* h, int member, fdf_handle** out) {
    if (!out) return FDF_ERR_ARG;
    return eguarded(h, [&](fdf::Ensemble& e) {
        fdf::Solver& s = e.member(member);
        fdf_handle* m = new fdf_handle;
        m->s = &s;
        m->borrowed = true;
        *out = m;
    });
}

int fdf_ensemble_run(fdf_ensemble* h, int nsteps) {
    if (nsteps < 0) return FDF_ERR_ARG;
    return eguarded(h, [&](fdf::Ensemble& e) { e.run(nsteps); });
}

int fdf_ensemble_time_steps(fdf_ensemble* h, int nsteps, double* ms) {
    if (nsteps < 0 || !ms) return FDF_ERR_ARG;
    return eguarded(h, [&](fdf::Ensemble& e) { *ms = e.time_steps(nsteps); });
}

int fdf_ensemble_autotune(fdf_ensemble* h, int steps, int* threads, long long* tile) {
    return eguarded(h, [&](fdf::Ensemble& e) {
        const fdf::EnsConfig c = e.autotune(steps);
        if (threads) *threads = c.threads;
        if (tile) *tile = c.tile;
    });
}

int fdf_ensemble_set_config(fdf_ensemble* h, int threads, long long tile) {
    return eguarded(h, [&](fdf::Ensemble& e) {
        fdf::EnsConfig c;
        c.threads = threads;
        c.tile = tile;
        e.set_config(c);
    });
}

int fdf_ensemble_use_graph(fdf_ensemble* h, int on) {
    return eguarded(h, [&](fdf::Ensemble& e) { e.use_graph(on != 0); });
}

int fdf_ensemble_node_stages(fdf_ensemble* h, long long* per_step) {
    if (!per_step) return FDF_ERR_ARG;
    return eguarded(h, [&](fdf::Ensemble& e) { *per_step = e.node_stages_per_step(); });
}

int fdf_ensemble_check_status(fdf_ensemble* h) {
    return eguarded(h, [&](fdf::Ensemble& e) { e.check_status(); });
}

const char* fdf_ensemble_last_error(fdf_ensemble* h) {
    if (!h) return g_create_error.c_str();
    return h->err.c_str();
}

const char* fdf_last_error(fdf_handle* h) {
    if (!h) return g_create_error.c_str();
    return h->err.c_str();
}

}  // extern "C"
