// TEST INFRASTRUCTURE — not product code.
//
// Compiles the reference ALMA engine (src/physics_engine.cpp of
// noira-913/Protein-Structure-Analysis) unmodified, from where it lies, and
// appends a plain C-ABI so the test suite and the CPU baseline can call the
// reference's own static kernels (NeighborList::build, born_radii,
// update_born, sasa_nonpolar, total_e, pair_e, ...) on numpy arrays.
//
// The translation unit is built by oracle/Makefile into
// oracle/_ref/protein_physics<EXT_SUFFIX>.  Because the reference's own
// PYBIND11_MODULE is compiled in as well, the same .so imports as the
// reference Python module `protein_physics` (its stock public API, used by
// the reference arm of bench.py) and loads via ctypes for the ref_* symbols.
//
// Only tests/, __graft_entry__.smoke() and bench.py's CPU-baseline leg may
// load this file's output, and only as the checker / the baseline.

// Pre-include everything the reference and pybind11 pull in, so the
// `private -> public` redefinition below touches only the reference's own
// classes (PhysicsEngine keeps its kernels private).
#include <algorithm>
#include <array>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <functional>
#include <map>
#include <memory>
#include <random>
#include <stdexcept>
#include <string>
#include <tuple>
#include <unordered_map>
#include <unordered_set>
#include <utility>
#include <vector>
#include <pybind11/pybind11.h>
#include <pybind11/stl.h>
#include <pybind11/numpy.h>
#ifdef _OPENMP
#include <omp.h>
#endif

#define private public
#include ALMA_REF_SRC
#undef private

namespace {

std::vector<Particle> make_particles(int n, const double* xyz, const double* q,
                                     const double* r, const double* eps) {
    std::vector<Particle> p;
    p.reserve((size_t)n);
    for (int i = 0; i < n; ++i)
        p.emplace_back(xyz[3 * i], xyz[3 * i + 1], xyz[3 * i + 2], q[i], r[i], eps[i], false);
    return p;
}

}  // namespace

extern "C" {

// ---- topology ---------------------------------------------------------------

void* ref_topo_build(int n, const char* const* resnames, const char* const* atomnames,
                     const int* res_idx) {
    auto* t = new BondTopology();
    std::vector<std::string> rn(resnames, resnames + n), an(atomnames, atomnames + n);
    std::vector<int> ri(res_idx, res_idx + n);
    t->build(rn, an, ri);
    return t;
}

void ref_topo_free(void* h) { delete static_cast<BondTopology*>(h); }

void ref_topo_add_disulfide(void* h, int i, int j) {
    static_cast<BondTopology*>(h)->add_disulfide(i, j);
}

void ref_topo_concerted_sidechain(void* h, int n, const double* xyz, double cutoff) {
    std::vector<double> z((size_t)n, 0.0);
    auto p = make_particles(n, xyz, z.data(), z.data(), z.data());
    static_cast<BondTopology*>(h)->identify_concerted_sidechain_pairs(p, cutoff);
}

// ---- neighbor list (physics_engine.cpp:293-342) ------------------------------

// Fills row_counts[n] and cols[] (reference cell-scan order).  Returns the
// total pair count, or -total when cap is too small (nothing written to cols).
int64_t ref_nl(int n, const double* xyz, int64_t* row_counts, int32_t* cols, int64_t cap) {
    std::vector<double> z((size_t)n, 0.0);
    auto p = make_particles(n, xyz, z.data(), z.data(), z.data());
    NeighborList nl;
    nl.build(p);
    int64_t tot = 0;
    for (int i = 0; i < n; ++i) tot += (int64_t)nl.nb[(size_t)i].size();
    if (tot > cap) return -tot;
    int64_t k = 0;
    for (int i = 0; i < n; ++i) {
        row_counts[i] = (int64_t)nl.nb[(size_t)i].size();
        for (size_t j : nl.nb[(size_t)i]) cols[k++] = (int32_t)j;
    }
    return tot;
}

// ---- Born radii / SASA / energy ----------------------------------------------

void ref_born_radii(int n, const double* xyz, const double* q, const double* r,
                    const double* eps, double* a_out) {
    auto p = make_particles(n, xyz, q, r, eps);
    NeighborList nl;
    nl.build(p);
    auto a = PhysicsEngine::born_radii(p, nl);
    std::copy(a.begin(), a.end(), a_out);
}

double ref_sasa(int n, const double* xyz, const double* q, const double* r, const double* eps) {
    auto p = make_particles(n, xyz, q, r, eps);
    NeighborList nl;
    nl.build(p);
    return PhysicsEngine::sasa_nonpolar(p, nl);
}

// terms_out[0..4] = {sasa, dihedral, disulfide, pair sum, total}.  The total
// is the reference's own calculate_potential(); the pair sum is total minus
// the three others.  topo may be NULL (no exclusions / dihedrals / SS).
double ref_energy(int n, const double* xyz, const double* q, const double* r,
                  const double* eps, void* topo_h, double* terms_out) {
    auto p = make_particles(n, xyz, q, r, eps);
    const BondTopology* topo = static_cast<const BondTopology*>(topo_h);
    PhysicsEngine eng;
    double total = eng.calculate_potential(p, topo);
    if (terms_out) {
        NeighborList nl;
        nl.build(p);
        double sasa = PhysicsEngine::sasa_nonpolar(p, nl);
        double dih = (topo && !topo->dihedrals.empty()) ? PhysicsEngine::dihedral_e(p, topo->dihedrals) : 0.0;
        double ss = (topo && !topo->disulfide_pairs.empty()) ? PhysicsEngine::ss_e(p, topo->disulfide_pairs) : 0.0;
        terms_out[0] = sasa;
        terms_out[1] = dih;
        terms_out[2] = ss;
        terms_out[3] = total - sasa - dih - ss;
        terms_out[4] = total;
    }
    return total;
}

double ref_pair_e(const double* pi6, const double* pj6, double ai, double aj) {
    Particle a(pi6[0], pi6[1], pi6[2], pi6[3], pi6[4], pi6[5]);
    Particle b(pj6[0], pj6[1], pj6[2], pj6[3], pj6[4], pj6[5]);
    return PhysicsEngine::pair_e(a, b, ai, aj);
}

// ---- one Metropolis proposal's ΔE, replayed without the RNG -----------------
//
// Replays the arithmetic of try_torsion (physics_engine.cpp:2328-2399) for
// kind == 0 (bond = rot-bond index) and of try_crankshaft (:2407-2501) for
// kind == 1 (bond = concerted-pair index), with the angle `delta` given
// instead of drawn.  State: the neighbor list and Born radii are rebuilt
// from `xyz` exactly as generate_ensemble does at chain start
// (:2288-2292).  The cross-pair sum restates the cross_e lambda
// (:2312-2323) line for line — it is a local lambda, not reachable from
// here.  Outputs: the four ΔE components {cross, sasa, dihedral, ss}, the
// post-move coordinates and Born radii (the proposal, before any
// Metropolis revert).  Returns the summed ΔE, or NaN for a degenerate
// proposal (empty side / zero-length axis), as the reference returns
// {false,false} there.
double ref_move_dE(int n, const double* xyz, const double* q, const double* r,
                   const double* eps, void* topo_h, int kind, int bond, double delta,
                   double* terms_out, double* new_xyz, double* new_a) {
    const BondTopology& topo = *static_cast<const BondTopology*>(topo_h);
    auto st = make_particles(n, xyz, q, r, eps);
    NeighborList nl;
    nl.build(st);
    auto a = PhysicsEngine::born_radii(st, nl);
    const size_t N = st.size();
    std::vector<bool> in_side(N, false);

    auto cross_e = [&]() -> double {
        double E = 0.0;
        for (size_t i = 0; i < N; ++i)
            for (size_t j : nl.nb[i]) {
                if (in_side[i] == in_side[j]) continue;
                if (topo.is_excluded((int)i, (int)j)) continue;
                double dx = st[i].x - st[j].x, dy = st[i].y - st[j].y, dz = st[i].z - st[j].z;
                if (dx * dx + dy * dy + dz * dz > PAIR_CUT2) continue;
                E += PhysicsEngine::pair_e(st[i], st[j], a[i], a[j]);
            }
        return E;
    };
    auto eval_terms = [&](double* out) {
        out[0] = cross_e();
        out[1] = PhysicsEngine::sasa_nonpolar(st, nl);
        out[2] = PhysicsEngine::dihedral_e_boundary(st, topo.dihedrals, in_side);
        out[3] = topo.disulfide_pairs.empty() ? 0.0
                                              : PhysicsEngine::ss_e_side(st, topo.disulfide_pairs, in_side);
    };

    const std::vector<int>* moved = nullptr;
    double before[4], after[4];
    const double nan = std::nan("");
    if (kind == 0) {
        const RotBond& rb = topo.rot_bonds[(size_t)bond];
        const std::vector<int>& side = topo.rot_bond_sides[(size_t)bond];
        if (side.empty()) return nan;
        double ax = st[rb.j].x - st[rb.i].x, ay = st[rb.j].y - st[rb.i].y, az = st[rb.j].z - st[rb.i].z;
        double al = std::sqrt(ax * ax + ay * ay + az * az);
        if (al < 1e-10) return nan;
        ax /= al; ay /= al; az /= al;
        double cosD = std::cos(delta), sinD = std::sin(delta);
        for (int k : side) in_side[(size_t)k] = true;
        eval_terms(before);
        double ox = st[rb.i].x, oy = st[rb.i].y, oz = st[rb.i].z;
        for (int k : side)
            PhysicsEngine::rodrigues(st[k].x, st[k].y, st[k].z, ox, oy, oz, ax, ay, az, cosD, sinD);
        for (int k : side) PhysicsEngine::update_born((size_t)k, st, nl, a);
        eval_terms(after);
        moved = &side;
    } else {
        int phi_k = topo.concerted_pairs[(size_t)bond].first;
        int psi_k = topo.concerted_pairs[(size_t)bond].second;
        const std::vector<int>& phi_side = topo.rot_bond_sides[(size_t)phi_k];
        const std::vector<int>& psi_side = topo.rot_bond_sides[(size_t)psi_k];
        if (phi_side.empty() || psi_side.empty()) return nan;
        for (int k : phi_side) in_side[(size_t)k] = true;
        const RotBond& phi_rb = topo.rot_bonds[(size_t)phi_k];
        double p1ox = st[phi_rb.i].x, p1oy = st[phi_rb.i].y, p1oz = st[phi_rb.i].z;
        double p1ax = st[phi_rb.j].x - p1ox, p1ay = st[phi_rb.j].y - p1oy, p1az = st[phi_rb.j].z - p1oz;
        double p1l = std::sqrt(p1ax * p1ax + p1ay * p1ay + p1az * p1az);
        if (p1l < 1e-10) return nan;
        p1ax /= p1l; p1ay /= p1l; p1az /= p1l;
        eval_terms(before);
        double cosD = std::cos(delta), sinD = std::sin(delta);
        for (int k : phi_side)
            PhysicsEngine::rodrigues(st[k].x, st[k].y, st[k].z, p1ox, p1oy, p1oz, p1ax, p1ay, p1az, cosD, sinD);
        const RotBond& psi_rb = topo.rot_bonds[(size_t)psi_k];
        double p2ox = st[psi_rb.i].x, p2oy = st[psi_rb.i].y, p2oz = st[psi_rb.i].z;
        double p2ax = st[psi_rb.j].x - p2ox, p2ay = st[psi_rb.j].y - p2oy, p2az = st[psi_rb.j].z - p2oz;
        double p2l = std::sqrt(p2ax * p2ax + p2ay * p2ay + p2az * p2az);
        if (p2l < 1e-10) return nan;
        p2ax /= p2l; p2ay /= p2l; p2az /= p2l;
        for (int k : psi_side)
            PhysicsEngine::rodrigues(st[k].x, st[k].y, st[k].z, p2ox, p2oy, p2oz, p2ax, p2ay, p2az, cosD, -sinD);
        for (int k : phi_side) PhysicsEngine::update_born((size_t)k, st, nl, a);
        eval_terms(after);
        moved = &phi_side;
    }
    (void)moved;
    double dE = 0.0;
    for (int t = 0; t < 4; ++t) {
        if (terms_out) terms_out[t] = after[t] - before[t];
    }
    dE = (after[0] - before[0]) + (after[1] - before[1]) + (after[2] - before[2]) + (after[3] - before[3]);
    if (new_xyz)
        for (size_t i = 0; i < N; ++i) {
            new_xyz[3 * i] = st[i].x;
            new_xyz[3 * i + 1] = st[i].y;
            new_xyz[3 * i + 2] = st[i].z;
        }
    if (new_a) std::copy(a.begin(), a.end(), new_a);
    return dE;
}

int ref_num_threads() {
    PhysicsEngine eng;
    return eng.num_threads();
}

}  // extern "C"
