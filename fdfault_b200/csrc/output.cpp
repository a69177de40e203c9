// Output units and fronts (see output.hpp).  Index clipping, field numbering
// and file contents follow src/outputunit.cpp:13-889, src/outputlist.cpp:11-113,
// src/front.cpp:17-359 and src/frontlist.cpp:11-109 for one process.
#include "output.hpp"

#include <cstring>
#include <fstream>
#include <stdexcept>

#include "kernels.hpp"
#include "solver.hpp"

namespace fdf {

namespace {

const char* kVol3[] = {"vx", "vy", "vz", "sxx", "sxy", "sxz", "syy", "syz", "szz", "lambda", "gammap",
                       "epxx", "epxy", "epxz", "epyy", "epyz", "epzz"};
const char* kVol2m2[] = {"vx", "vy", "sxx", "sxy", "syy", "szz", "lambda", "gammap",
                         "epxx", "epxy", "epxz", "epyy", "epyz", "epzz"};
const char* kVol2m3[] = {"vz", "sxz", "syz", "lambda", "gammap", "epxx", "epxy", "epxz", "epyy", "epyz", "epzz"};
const char* kIf3[] = {"Vx", "Vy", "Vz", "V", "Ux", "Uy", "Uz", "U", "Sx", "Sy", "Sz", "S", "Sn", "state"};
const char* kIf2m2[] = {"Vx", "Vy", "V", "Ux", "Uy", "U", "Sx", "Sy", "S", "Sn", "state"};
const char* kIf2m3[] = {"Vz", "V", "Uz", "U", "Sz", "S", "Sn", "state"};

int find_name(const char* const* list, int n, const std::string& s) {
    for (int i = 0; i < n; i++)
        if (s == list[i]) return i;
    return -1;
}

bool is_volume(const std::string& f) {
    return find_name(kVol3, 17, f) >= 0;
}

void write_meta(const std::string& base, const std::string& field, int ntout, const int nx[3]) {
    std::ofstream m(base + ".m");
    if (!m) throw std::runtime_error("Error writing parameters to matlab file");
    m << "endian = 'l';\n";
    if (!field.empty()) m << "field = '" << field << "';\n";
    if (ntout >= 0) m << "nt = " << ntout << ";\n";
    m << "nx = " << nx[0] << ";\n";
    m << "ny = " << nx[1] << ";\n";
    if (nx[2] >= 0) m << "nz = " << nx[2] << ";\n";
    std::ofstream p(base + ".py");
    if (!p) throw std::runtime_error("Error writing parameters to python file");
    p << "endian = '<'\n";
    if (!field.empty()) p << "field = '" << field << "';\n";
    if (ntout >= 0) p << "nt = " << ntout << "\n";
    p << "nx = " << nx[0] << "\n";
    p << "ny = " << nx[1] << "\n";
    if (nx[2] >= 0) p << "nz = " << nx[2] << "\n";
}

}  // namespace

OutputList::OutputList(Solver& s) : S_(s) {
    const ProblemSpec& P = s.spec();
    const Layout& L = s.layout();
    const int ndim = P.ndim, mode = P.mode;
    for (const OutputSpec& o : P.outputs) {
        Unit u;
        u.name = o.name;
        u.field = o.field;
        if (!(o.ts > 0) || !(o.tp >= o.tm)) throw std::runtime_error("invalid output time range for " + o.name);
        for (int i = 0; i < 3; i++)
            if (!(o.xm[i] < P.nx[i]) || !(o.xs[i] > 0) || !(o.xp[i] >= o.xm[i]))
                throw std::runtime_error("invalid output index range for " + o.name);
        if ((o.field == "lambda" || o.field == "gammap") && !P.plastic())
            throw std::runtime_error("plastic output field requires plastic material");
        if (o.field.size() == 4 && o.field.compare(0, 2, "ep") == 0 && !P.plastic_tensor)
            throw std::runtime_error("plastic strain output requires plastic_tensor");
        if (ndim == 2 && mode == 2 && o.field == "szz" && !P.plastic())
            throw std::runtime_error("szz output in mode II requires plastic material");
        if (is_volume(o.field)) {
            u.location = -1;
        } else {
            u.location = -1;
            const auto& ifs = s.ifaces();
            for (size_t i = 0; i < ifs.size(); i++) {
                const IfaceSpec& I = P.ifaces[i];
                const IfaceDev& D = ifs[i];
                const BlockDev& B2 = s.blocks()[D.b2];
                int ixm[3], ixp[3];
                for (int k = 0; k < 3; k++) {
                    ixm[k] = B2.lo[k];
                    ixp[k] = B2.lo[k] + B2.n[k] - 1;
                }
                ixp[I.direction] = B2.lo[I.direction];
                int d = I.direction, a = (d == 0) ? 1 : 0, b = (d == 2) ? 1 : 2;
                if (o.xm[d] == o.xp[d] && (o.xm[d] == ixm[d] || o.xm[d] == ixm[d] - 1) && o.xm[a] >= ixm[a] &&
                    o.xm[a] <= ixp[a] && o.xm[b] >= ixm[b] && o.xm[b] <= ixp[b]) {
                    u.location = (int)i;
                    break;
                }
            }
            if (u.location == -1)
                throw std::runtime_error("Could not find interface corresponding to input indices for " + o.name);
            if (s.ifaces()[u.location].kind < 1) throw std::runtime_error("Interface for output is not frictional");
            if (o.field == "state" && s.ifaces()[u.location].kind != 3)
                throw std::runtime_error("Interface for output does not have a state variable");
        }
        // field index (outputunit.cpp:120-277)
        int f = -1;
        if (ndim == 3)
            f = (u.location == -1) ? find_name(kVol3, 17, o.field) : find_name(kIf3, 14, o.field);
        else if (mode == 2)
            f = (u.location == -1) ? find_name(kVol2m2, 14, o.field) : find_name(kIf2m2, 11, o.field);
        else
            f = (u.location == -1) ? find_name(kVol2m3, 11, o.field) : find_name(kIf2m3, 8, o.field);
        if (f < 0) throw std::runtime_error("Error in specifying output field " + o.field);
        u.fidx = f;
        // time limits
        u.tm = o.tm < 0 ? 0 : o.tm;
        u.tp = o.tp > s.nt() ? s.nt() : o.tp;
        u.tp = u.tp - (u.tp - u.tm) % o.ts;
        u.ts = o.ts;
        // spatial limits
        int ixm[3] = {0, 0, 0}, ixp[3] = {0, 0, 0};
        if (u.location >= 0) {
            const IfaceDev& D = s.ifaces()[u.location];
            const BlockDev& B2 = s.blocks()[D.b2];
            for (int k = 0; k < 3; k++) {
                ixm[k] = B2.lo[k];
                ixp[k] = B2.lo[k] + B2.n[k] - 1;
            }
            ixp[D.direction] = B2.lo[D.direction];
        }
        for (int i = 0; i < 3; i++) {
            if (u.location == -1) {
                u.xm[i] = o.xm[i] < 0 ? 0 : o.xm[i];
                u.xp[i] = (o.xp[i] >= P.nx[i]) ? P.nx[i] - 1 : o.xp[i] - (o.xp[i] - o.xm[i]) % o.xs[i];
            } else {
                u.xm[i] = o.xm[i] < ixm[i] ? ixm[i] : o.xm[i];
                u.xp[i] = (o.xp[i] > ixp[i]) ? ixp[i] : o.xp[i] - (o.xp[i] - o.xm[i]) % o.xs[i];
                if (u.xm[i] > u.xp[i]) u.xp[i] = u.xm[i];
            }
            u.xs[i] = o.xs[i];
            u.nx[i] = (u.xp[i] - u.xm[i]) / u.xs[i] + 1;
        }
        if (ndim == 2) {
            u.xm[2] = 0;
            u.xp[2] = 0;
            u.xs[2] = 1;
            u.nx[2] = 1;
        }
        for (int i = 0; i < 3; i++)
            if (u.nx[i] == 1) u.xs[i] = 1;
        // data source
        if (u.location == -1) {
            u.comp = f;
            if (f >= L.nv && f < L.nv + L.ns && s.precision() == 0) needs_abs_ = true;
        } else {
            const int dir = s.ifaces()[u.location].direction;
            const long long nn = (long long)s.ifaces()[u.location].n0 * s.ifaces()[u.location].n1;
            if (ndim == 3) {
                // 0-2 vx, 3 v, 4-6 ux, 7 u, 8-10 sx, 11 s, 12 sn, 13 state
                int grp = (f <= 2) ? 7 : (f == 3) ? 2 : (f <= 6) ? 5 : (f == 7) ? 0 : (f <= 10) ? 8 : (f == 11) ? 3 : (f == 12) ? 4 : 9;
                u.comp = grp;
                if (f <= 2 || (f >= 4 && f <= 6) || (f >= 8 && f <= 10)) {
                    int c = (f <= 2) ? f : (f <= 6 ? f - 4 : f - 8);
                    int t0 = (dir == 0) ? 1 : 0, t1 = (dir == 2) ? 1 : 2;
                    if (c == t0)
                        u.offset = 0;
                    else if (c == t1)
                        u.offset = nn;
                    else
                        throw std::runtime_error("Field not associated with this interface");
                }
            } else if (mode == 2) {
                // 0-1 vx, 2 v, 3-4 ux, 5 u, 6-7 sx, 8 s, 9 sn, 10 state
                int grp = (f <= 1) ? 7 : (f == 2) ? 2 : (f <= 4) ? 5 : (f == 5) ? 0 : (f <= 7) ? 8 : (f == 8) ? 3 : (f == 9) ? 4 : 9;
                u.comp = grp;
                if (f <= 1 || f == 3 || f == 4 || f == 6 || f == 7) {
                    int c = (f <= 1) ? f : (f <= 4 ? f - 3 : f - 6);
                    if (c == dir) throw std::runtime_error("Field not associated with this interface");
                }
            } else {
                int grp = (f == 0) ? 7 : (f == 1) ? 2 : (f == 2) ? 5 : (f == 3) ? 0 : (f == 4) ? 8 : (f == 5) ? 3 : (f == 6) ? 4 : 9;
                u.comp = grp;
            }
        }
        open_unit(u);
        units_.push_back(u);
    }
}

void OutputList::open_unit(Unit& u) {
    const ProblemSpec& P = S_.spec();
    const std::string base = P.datadir + P.name + "_" + u.name;
    u.data = std::fopen((base + "_" + u.field + ".dat").c_str(), "wb");
    if (!u.data) throw std::runtime_error("Error opening file " + base + "_" + u.field + ".dat");
    // grid coordinates of the output points
    const size_t nall = (size_t)P.nx[0] * P.nx[1] * P.nx[2];
    std::vector<double> x(nall);
    static const char* xyz[3] = {"x", "y", "z"};
    for (int c = 0; c < P.ndim; c++) {
        S_.get_geometry(0, c, x.data());
        FILE* fx = std::fopen((base + "_" + xyz[c] + ".dat").c_str(), "wb");
        if (!fx) throw std::runtime_error("Error opening file in outputunit");
        for (int i = 0; i < u.nx[0]; i++)
            for (int j = 0; j < u.nx[1]; j++)
                for (int k = 0; k < u.nx[2]; k++) {
                    size_t id = ((size_t)(u.xm[0] + i * u.xs[0]) * P.nx[1] + (u.xm[1] + j * u.xs[1])) * P.nx[2] +
                                (u.xm[2] + k * u.xs[2]);
                    std::fwrite(&x[id], sizeof(double), 1, fx);
                }
        std::fclose(fx);
    }
    if (u.tp > u.tm) {
        u.tfile = std::fopen((base + "_t.dat").c_str(), "wb");
        if (!u.tfile) throw std::runtime_error("Error opening file in outputunit");
    }
    write_meta(base, u.field, (u.tp - u.tm) / u.ts + 1, u.nx);
}

void OutputList::enqueue(Unit& u, int tstep, double* dst) {
    Solver& S = S_;
    OutWindow w;
    for (int i = 0; i < 3; i++) {
        w.xm[i] = u.xm[i];
        w.xs[i] = u.xs[i];
        w.n[i] = u.nx[i];
    }
    if (u.location == -1) {
        const Layout& L = S.L_;
        const int comp = u.comp;
        const bool stress = comp >= L.nv && comp < L.nv + L.ns;
        if (stress && S.precision_ == 0 && tstep > 0 && S.ABS_) {
            // absolute stresses of the step as the reference's output round trip left them
            launch_gather_window<double>(L, S.ABS_, comp - L.nv, 0, S.P_.s0, nullptr, w, dst, S.stream_);
        } else {
            const bool plastic_field = comp >= L.nfields;
            void* base = plastic_field ? S.FP_ : S.F_[S.cur_];
            const int c = plastic_field ? comp - L.nfields : comp;
            if (S.precision_ == 0)
                launch_gather_window<double>(L, (const double*)base, c, !plastic_field, S.P_.s0, S.S_, w, dst,
                                             S.stream_);
            else
                launch_gather_window<float>(L, (const float*)base, c, !plastic_field, S.P_.s0, S.S_, w, dst,
                                            S.stream_);
        }
    } else {
        const IfaceDev& D = S.ifaces()[u.location];
        const int dir = D.direction;
        const int a = (dir == 0) ? 1 : 0, b = (dir == 2) ? 1 : 2;
        launch_gather_fault(S.fault_ptr(u.location, u.comp), u.offset, D.n1, a, b, D.mlb[a], D.mlb[b], w, dst,
                            S.stream_);
    }
}

void OutputList::flush(int slot) {
    Slot& sl = slots_[slot];
    if (!sl.pending) return;
    if (cudaEventSynchronize(sl.done) != cudaSuccess) throw std::runtime_error("CUDA error waiting for output copy");
    const double* h = hstage_ + (size_t)slot * cap_;
    for (const auto& it : sl.items) {
        Unit& u = units_[it.first];
        if (u.tfile) {
            const double t = (double)sl.tstep * S_.dt();
            std::fwrite(&t, sizeof(double), 1, u.tfile);
        }
        const size_t n = (size_t)u.nx[0] * u.nx[1] * u.nx[2];
        if (std::fwrite(h + it.second, sizeof(double), n, u.data) != n)
            throw std::runtime_error("Error writing output unit " + u.name);
    }
    sl.pending = false;
    sl.items.clear();
}

void OutputList::write(int tstep) {
    std::vector<std::pair<int, size_t>> due;
    size_t n = 0;
    for (size_t i = 0; i < units_.size(); i++) {
        const Unit& u = units_[i];
        if (tstep < u.tm || tstep > u.tp || (tstep - u.tm) % u.ts != 0) continue;
        due.push_back({(int)i, n});
        n += (size_t)u.nx[0] * u.nx[1] * u.nx[2];
    }
    if (due.empty()) return;
    if (!dstage_) {   // every unit's window fits in one slot
        for (const Unit& u : units_) cap_ += (size_t)u.nx[0] * u.nx[1] * u.nx[2];
        if (cudaMalloc(&dstage_, 2 * cap_ * sizeof(double)) != cudaSuccess ||
            cudaMallocHost(&hstage_, 2 * cap_ * sizeof(double)) != cudaSuccess)
            throw std::runtime_error("CUDA error allocating output staging");
        for (Slot& sl : slots_)
            if (cudaEventCreateWithFlags(&sl.done, cudaEventDisableTiming) != cudaSuccess)
                throw std::runtime_error("CUDA error creating output event");
    }
    const int slot = next_;
    flush(slot);   // the slot's previous contents (two output steps ago) go to the files first
    double* d = dstage_ + (size_t)slot * cap_;
    for (const auto& it : due) enqueue(units_[it.first], tstep, d + it.second);
    cudaStream_t st = S_.stream();
    if (cudaMemcpyAsync(hstage_ + (size_t)slot * cap_, d, n * sizeof(double), cudaMemcpyDeviceToHost, st) !=
            cudaSuccess ||
        cudaEventRecord(slots_[slot].done, st) != cudaSuccess)
        throw std::runtime_error("CUDA error queueing output copy");
    slots_[slot].tstep = tstep;
    slots_[slot].items = due;
    slots_[slot].pending = true;
    next_ = 1 - slot;
}

void OutputList::close() {
    if (closed_) return;
    closed_ = true;
    flush(next_);       // the older slot first, then the newer
    flush(1 - next_);
    for (Unit& u : units_) {
        if (u.tfile) std::fclose(u.tfile);
        if (u.data) std::fclose(u.data);
        u.tfile = u.data = nullptr;
    }
    const ProblemSpec& P = S_.spec();
    if (!P.front_on) return;
    const size_t nall = (size_t)P.nx[0] * P.nx[1] * P.nx[2];
    std::vector<double> x;
    static const char* xyz[3] = {"x", "y", "z"};
    for (size_t n = 0; n < S_.ifaces().size(); n++) {
        const IfaceDev& D = S_.ifaces()[n];
        if (D.kind < 1) continue;
        const std::string base = P.datadir + P.name + "_front_" + std::to_string(n);
        const size_t nn = (size_t)D.n0 * D.n1;
        std::vector<double> tv(nn);
        S_.get_fault((int)n, 12, tv.data());
        FILE* ft = std::fopen((base + "_t.dat").c_str(), "wb");
        if (!ft) throw std::runtime_error("Error opening file in front");
        std::fwrite(tv.data(), sizeof(double), nn, ft);
        std::fclose(ft);
        const int dir = D.direction, a = (dir == 0) ? 1 : 0, b = (dir == 2) ? 1 : 2;
        if (x.size() != nall) x.resize(nall);
        for (int c = 0; c < P.ndim; c++) {
            S_.get_geometry(0, c, x.data());
            FILE* fx = std::fopen((base + "_" + xyz[c] + ".dat").c_str(), "wb");
            if (!fx) throw std::runtime_error("Error opening file in front");
            for (int i = 0; i < D.n0; i++)
                for (int j = 0; j < D.n1; j++) {
                    int pos[3] = {D.mlb[0], D.mlb[1], D.mlb[2]};
                    pos[dir] += 1;   // the plus-side plane (front.cpp uses the data2 side)
                    pos[a] += i;
                    pos[b] += j;
                    size_t id = ((size_t)pos[0] * P.nx[1] + pos[1]) * P.nx[2] + pos[2];
                    std::fwrite(&x[id], sizeof(double), 1, fx);
                }
            std::fclose(fx);
        }
        int nx3[3] = {D.n0, D.n1, -1};
        write_meta(base, "", -1, nx3);
    }
}

OutputList::~OutputList() {
    for (Unit& u : units_) {
        if (u.tfile) std::fclose(u.tfile);
        if (u.data) std::fclose(u.data);
    }
    for (Slot& sl : slots_)
        if (sl.done) cudaEventDestroy(sl.done);
    if (dstage_) cudaFree(dstage_);
    if (hstage_) cudaFreeHost(hstage_);
}

}  // namespace fdf
