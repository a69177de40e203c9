// Reader for the fdfault .in format (see input.hpp).  Section readers follow
// src/problem.cpp:24-50, src/domain.cpp:35-76, src/fields.cpp:24-47,
// src/block.cpp:52-107, src/interface.cpp:28-54, src/friction.cpp:76-129,
// src/slipweak.cpp:42-96, src/stz.cpp:51-113, src/outputlist.cpp:28-72 and
// src/frontlist.cpp:20-40 of the reference.
#include "input.hpp"

#include <cstdlib>
#include <fstream>
#include <sstream>
#include <stdexcept>

namespace fdf {

namespace {

// Token stream positioned after a header line, mirroring `paramfile >> x`.
class Section {
  public:
    Section(const std::string& file, const std::string& header, const std::string& after = "")
        : in_(file) {
        if (!in_.is_open()) throw std::runtime_error("Error opening input file " + file);
        std::string line;
        if (!after.empty()) {
            bool seen = false;
            while (std::getline(in_, line))
                if (line == after) {
                    seen = true;
                    break;
                }
            if (!seen) return;
        }
        while (std::getline(in_, line))
            if (line == header) {
                found_ = true;
                return;
            }
    }
    bool found() const { return found_; }
    std::string str() {
        std::string s;
        if (!(in_ >> s)) throw std::runtime_error("unexpected end of input while reading a section");
        return s;
    }
    double dbl() { return std::strtod(str().c_str(), nullptr); }
    int integer() { return static_cast<int>(std::strtol(str().c_str(), nullptr, 10)); }
    std::ifstream& stream() { return in_; }

  private:
    std::ifstream in_;
    bool found_ = false;
};

PertSpec read_pert(Section& s, int nval) {
    PertSpec p;
    std::string ty = s.str();
    p.type = pert_type_code(ty);
    if (p.type < 0) throw std::runtime_error("unknown perturbation type " + ty);
    p.t0 = s.dbl();
    p.x0 = s.dbl();
    p.dx = s.dbl();
    p.y0 = s.dbl();
    p.dy = s.dbl();
    for (int k = 0; k < nval; k++) p.val[k] = s.dbl();
    if (p.t0 < 0. || p.dx < 0. || p.dy < 0.) throw std::runtime_error("invalid perturbation parameters");
    return p;
}

}  // namespace

int pert_type_code(const std::string& s) {
    if (s == "constant") return 0;
    if (s == "gaussian") return 1;
    if (s == "ellipse") return 2;
    if (s == "linear") return 3;
    if (s == "boxcar") return 4;
    return -1;
}

ProblemSpec read_problem(const std::string& infile) {
    ProblemSpec P;
    P.infile = infile;
    {
        Section s(infile, "[fdfault.problem]");
        if (!s.found()) throw std::runtime_error("Error reading problem from input file");
        P.name = s.str();
        P.datadir = s.str();
        P.nt = s.integer();
        P.dt = s.dbl();
        P.ttot = s.dbl();
        P.cfl = s.dbl();
        P.ninfo = s.integer();
        P.rkorder = s.integer();
    }
    std::vector<std::string> iftype;
    {
        Section s(infile, "[fdfault.domain]");
        if (!s.found()) throw std::runtime_error("Error reading domain from input file");
        P.ndim = s.integer();
        P.mode = s.integer();
        for (int i = 0; i < 3; i++) P.nx[i] = s.integer();
        for (int i = 0; i < 3; i++) P.nblocks[i] = s.integer();
        for (int i = 0; i < 3; i++) {
            if (P.nblocks[i] <= 0 || P.nblocks[i] > FDF_MAX_BLOCKS_PER_DIM)
                throw std::runtime_error("invalid number of blocks");
            P.nx_block[i].resize(P.nblocks[i]);
            for (int j = 0; j < P.nblocks[i]; j++) P.nx_block[i][j] = s.integer();
        }
        int nif = s.integer();
        if (nif < 0) throw std::runtime_error("invalid number of interfaces");
        for (int i = 0; i < nif; i++) iftype.push_back(s.str());
        P.sbporder = s.integer();
        P.material = s.str();
    }
    if (!(P.ndim == 2 || P.ndim == 3)) throw std::runtime_error("ndim must be 2 or 3");
    if (!(P.mode == 2 || P.mode == 3)) throw std::runtime_error("mode must be 2 or 3");
    if (!(P.material == "elastic" || P.material == "plastic")) throw std::runtime_error("invalid material");
    if (!(P.sbporder >= 2 && P.sbporder <= 4)) throw std::runtime_error("sbporder must be 2, 3 or 4");
    if (P.ndim == 2 && P.nx[2] != 1) throw std::runtime_error("2D problems need nz = 1");
    for (int i = 0; i < 3; i++) {
        int sum = 0;
        P.xm_block[i].resize(P.nblocks[i]);
        for (int j = 0; j < P.nblocks[i]; j++) {
            P.xm_block[i][j] = sum;
            sum += P.nx_block[i][j];
        }
        if (sum != P.nx[i] || P.nx[i] <= 0) throw std::runtime_error("block sizes do not sum to the domain size");
    }
    {
        Section s(infile, "[fdfault.fields]");
        if (!s.found()) throw std::runtime_error("Error reading fields from input file");
        for (int i = 0; i < 6; i++) P.s0[i] = s.dbl();
        P.loadfile = s.str();
        P.matfile = s.str();
        P.plastic_tensor = s.integer() != 0;
    }
    if (P.matfile != "none" && P.ndim == 2 && P.mode == 3)
        // the reference's time step reads a third material array that mode III
        // does not have (block.cpp:387-388 with nmat = 2, fields.cpp:58-61)
        throw std::runtime_error("heterogeneous material files are not supported for mode III");
    {
        Section s(infile, "[fdfault.operator]");
        P.cdiss = s.found() ? s.dbl() : 0.0;
    }
    int nbt = P.nblockstot();
    if (nbt > FDF_MAX_BLOCKS) throw std::runtime_error("too many blocks");
    P.blocks.resize(nbt);
    for (int i = 0; i < P.nblocks[0]; i++)
        for (int j = 0; j < P.nblocks[1]; j++)
            for (int k = 0; k < P.nblocks[2]; k++) {
                BlockSpec& b = P.blocks[(i * P.nblocks[1] + j) * P.nblocks[2] + k];
                b.coords[0] = i;
                b.coords[1] = j;
                b.coords[2] = k;
                std::ostringstream hdr;
                hdr << "[fdfault.block" << i << j << k << "]";
                Section s(infile, hdr.str());
                if (!s.found()) throw std::runtime_error("Error reading block " + hdr.str() + " from input file");
                b.rho = s.dbl();
                b.lam = s.dbl();
                b.g = s.dbl();
                if (P.plastic()) {
                    b.mu = s.dbl();
                    b.coh = s.dbl();
                    b.beta = s.dbl();
                    b.eta = s.dbl();
                }
                for (int d = 0; d < P.ndim; d++) b.xb[d] = s.dbl();
                for (int d = 0; d < P.ndim; d++) b.lb[d] = s.dbl();
                for (int f = 0; f < 2 * P.ndim; f++) b.btype[f] = s.str();
                for (int f = 0; f < 2 * P.ndim; f++) b.bfile[f] = s.str();
                int c[3] = {i, j, k};
                for (int d = 0; d < 3; d++) {
                    b.nx[d] = (d < P.ndim) ? P.nx_block[d][c[d]] : 1;
                    b.xm[d] = (d < P.ndim) ? P.xm_block[d][c[d]] : 0;
                    if (d < P.ndim && b.nx[d] < 4 * P.sbporder - 3)
                        throw std::runtime_error("block has too few points for the finite difference operator");
                }
                if (!(b.rho > 0 && b.lam > 0 && b.g > 0)) throw std::runtime_error("material properties must be positive");
                for (int f = 0; f < 2 * P.ndim; f++)
                    if (!(b.btype[f] == "none" || b.btype[f] == "absorbing" || b.btype[f] == "free" ||
                          b.btype[f] == "rigid"))
                        throw std::runtime_error("invalid boundary type " + b.btype[f]);
            }
    for (size_t n = 0; n < iftype.size(); n++) {
        IfaceSpec I;
        I.kind = iftype[n];
        if (!(I.kind == "locked" || I.kind == "frictionless" || I.kind == "slipweak" || I.kind == "stz"))
            throw std::runtime_error("invalid interface type " + I.kind);
        std::ostringstream hs;
        hs << "[fdfault.interface" << n << "]";
        const std::string hdr = hs.str();
        {
            Section s(infile, hdr);
            if (!s.found()) throw std::runtime_error("Error reading interface " + std::to_string(n) + " from input file");
            std::string dir = s.str();
            if (dir == "x")
                I.direction = 0;
            else if (dir == "y")
                I.direction = 1;
            else if (dir == "z" && P.ndim == 3)
                I.direction = 2;
            else
                throw std::runtime_error("invalid interface direction " + dir);
            for (int i = 0; i < 3; i++) I.idx1[i] = s.integer();
            for (int i = 0; i < 3; i++) I.idx2[i] = s.integer();
            for (int i = 0; i < 3; i++) {
                int want = I.idx1[i] + (i == I.direction ? 1 : 0);
                if (I.idx2[i] != want || I.idx1[i] < 0 || I.idx2[i] >= P.nblocks[i])
                    throw std::runtime_error("interface must join adjacent blocks");
            }
        }
        if (I.kind != "locked") {
            Section s(infile, "[fdfault.friction]", hdr);
            if (!s.found()) throw std::runtime_error("Error reading interface " + std::to_string(n) + " from input file");
            int nl = s.integer();
            for (int l = 0; l < nl; l++) {
                PertSpec p = read_pert(s, 3);
                if (P.ndim == 2 && P.mode == 2) p.val[2] = 0.;
                if (P.ndim == 2 && P.mode == 3) p.val[1] = 0.;
                I.loads.push_back(p);
            }
            I.loadfile = s.str();
        }
        if (I.kind == "slipweak") {
            Section s(infile, "[fdfault.slipweak]", hdr);
            if (!s.found()) throw std::runtime_error("Error reading slipweak from input file");
            int np = s.integer();
            for (int l = 0; l < np; l++) I.perts.push_back(read_pert(s, 6));
            I.paramfile = s.str();
        } else if (I.kind == "stz") {
            Section s(infile, "[fdfault.stz]", hdr);
            if (!s.found()) throw std::runtime_error("Error reading stz from input file");
            I.chi0 = s.dbl();
            I.statefile = s.str();
            int np = s.integer();
            for (int l = 0; l < np; l++) I.perts.push_back(read_pert(s, 9));
            I.paramfile = s.str();
        }
        P.ifaces.push_back(I);
    }
    if ((int)P.ifaces.size() > FDF_MAX_IFACES) throw std::runtime_error("too many interfaces");
    {
        Section s(infile, "[fdfault.outputlist]");
        if (s.found()) {
            std::ifstream& in = s.stream();
            std::string line;
            while (std::getline(in, line)) {
                if (line.empty()) break;
                OutputSpec o;
                o.name = line;
                in >> o.field >> o.tm >> o.tp >> o.ts;
                for (int i = 0; i < 3; i++) in >> o.xm[i] >> o.xp[i] >> o.xs[i];
                std::getline(in, line);
                if (!in) throw std::runtime_error("Error reading outputlist from input file");
                P.outputs.push_back(o);
            }
        }
    }
    {
        Section s(infile, "[fdfault.frontlist]");
        if (s.found()) {
            P.front_on = s.integer() != 0;
            if (P.front_on) {
                P.front_field = s.str();
                P.front_value = s.dbl();
                if (!(P.front_field == "V" || P.front_field == "U") || !(P.front_value > 0.))
                    throw std::runtime_error("invalid front parameters");
            }
        }
    }
    return P;
}

}  // namespace fdf
