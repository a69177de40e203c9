// Output units and rupture fronts in the reference's on-disk layout, so the
// fdfault Python and MATLAB readers load them unchanged:
//   {datadir}{problem}_{unit}_{field}.dat   f8, native endian, C order (t, x, y, z)
//   {datadir}{problem}_{unit}_{x|y|z}.dat   grid coordinates of the output points
//   {datadir}{problem}_{unit}_t.dat         output times (when the window has >1 step)
//   {datadir}{problem}_{unit}.m / .py       sizes and endianness
//   {datadir}{problem}_front_{n}_t.dat (+ _x/_y/_z, .m, .py) first times V >= threshold
// Semantics follow src/outputunit.cpp:13-889 and src/front.cpp:17-359 for a
// single process owning the whole grid.
//
// At an output step the due units' index windows are gathered on the device
// (with the absolute-stress conversion of the read-back) into one staging
// slot and copied to pinned host memory by one asynchronous copy on the
// solver stream; the files are written when the slot is needed again two
// output steps later, or at close, so the copies overlap the steps between.
#pragma once

#include <cuda_runtime.h>

#include <cstdio>
#include <string>
#include <vector>

namespace fdf {

class Solver;

class OutputList {
  public:
    explicit OutputList(Solver& s);
    ~OutputList();
    void write(int tstep);   // outputlist::write_list
    void close();            // outputlist::close_list + frontlist::write_list
    bool needs_abs_stress() const { return needs_abs_; }

  private:
    struct Unit {
        std::string name, field;
        int location = -1;   // -1 volume, else interface index
        int fidx = 0;        // field index in the reference's numbering
        int tm = 0, tp = 0, ts = 1;
        int xm[3] = {0, 0, 0}, xp[3] = {0, 0, 0}, xs[3] = {1, 1, 1}, nx[3] = {1, 1, 1};
        FILE* data = nullptr;
        FILE* tfile = nullptr;
        int comp = 0;        // volume component, or fault array selector
        long long offset = 0;   // offset of the tangential component in a 2-component fault array
    };
    void open_unit(Unit& u);
    void enqueue(Unit& u, int tstep, double* dst);   // gather u's window at this step into dst (device)
    void flush(int slot);                             // wait for a slot's copy and write its files
    Solver& S_;
    std::vector<Unit> units_;
    bool needs_abs_ = false;
    bool closed_ = false;
    // two staging slots (device + pinned host), each sized for every unit's window
    struct Slot {
        int tstep = -1;
        std::vector<std::pair<int, size_t>> items;   // (unit, offset in the slot)
        cudaEvent_t done = nullptr;
        bool pending = false;
    };
    Slot slots_[2];
    int next_ = 0;
    size_t cap_ = 0;
    double* dstage_ = nullptr;
    double* hstage_ = nullptr;
};

}  // namespace fdf
