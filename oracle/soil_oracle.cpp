// soil_oracle.cpp — CPU FP64 restatement of the SOIL substrate hot path.
//
// TEST INFRASTRUCTURE ONLY.  This file is the checker the CUDA path is
// compared against (tests/, __graft_entry__.smoke, bench.py's CPU baseline
// leg).  Nothing in the product links or calls it.
//
// The reference (SueHeir/soil) is Rust with unvendored `grass` git
// dependencies and cannot be built in this environment, so this is a
// function-by-function restatement of its single-rank periodic path.  Each
// function cites the reference file:line it follows (paths are inside the
// reference project).  Arithmetic is kept in the reference's operation
// order: Rust never contracts a*b+c, so this file is compiled with
// -ffp-contract=off and Rust's `mul_add` is std::fma.
//
// Pins: the reference's own known-answer tests (ported in
// tests/test_oracle_known_answers.py) and an O(N^2) periodic all-pairs
// equality check of the neighbor list (tests/test_oracle_allpairs.py).
//
// Scheduling assumptions about the unvendored `grass` scheduler: a run
// condition is evaluated when its system runs, and within one phase systems
// run in `.before` order, ties broken by registration order
// (crates/soil_core/src/schedule.rs:10-12) with the plugins added in the
// order Atom, Domain, Neighbor, Communication (examples/minimal_sim.rs:33-36).

#include <algorithm>
#include <array>
#include <cfloat>
#include <climits>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <string>
#include <vector>

#include "soil_cuda.h"

namespace {

using V3 = std::array<double, 3>;
using I3 = std::array<int32_t, 3>;

enum State { FULL_REBUILD = 0, COMMUNICATE_ONLY = 1 };

// Rust `f64 as i32`: saturating, NaN -> 0.
int32_t sat_i32(double v) {
    if (std::isnan(v)) return 0;
    if (v >= 2147483647.0) return INT32_MAX;
    if (v <= -2147483648.0) return INT32_MIN;
    return (int32_t)v;
}
int32_t clampi(int32_t v, int32_t lo, int32_t hi) { return v < lo ? lo : (v > hi ? hi : v); }
// Rust f64::round: half away from zero (same as C round()).
double rround(double v) { return std::round(v); }

struct Column {
    std::string name;
    int width;
    unsigned flags;
    std::vector<double> data;  // Vec<[f64; width]>: data[i*width + k]
};

struct Swap {  // SwapData, comm.rs:114-124
    std::vector<size_t> send_indices;
    size_t recv_start = 0, recv_count = 0;
    int to_proc = -1, from_proc = -1;
    V3 periodic_offset{0, 0, 0};
    V3 vel_offset{0, 0, 0};
};

struct Sys {
    // ---- Atom (atom.rs:406-431) ----
    uint32_t nlocal = 0, nghost = 0;
    double dt = 1.0;
    std::vector<uint32_t> tag, atom_type;
    std::vector<int32_t> origin_index;
    std::vector<uint8_t> is_ghost;
    std::vector<V3> pos, vel, force;
    std::vector<double> cutoff_radius, mass, inv_mass;
    std::vector<I3> image;
    std::vector<Column> cols;  // AtomDataRegistry stores, registration order

    // ---- Domain (domain.rs:105-142), single rank ----
    V3 blo{0, 0, 0}, bhi{1, 1, 1}, size{1, 1, 1};
    V3 sub_lo{0, 0, 0}, sub_hi{1, 1, 1}, sub_len{1, 1, 1};
    V3 sub_lam_lo{0, 0, 0}, sub_lam_hi{1, 1, 1};
    V3 tilt{0, 0, 0}, bvel{0, 0, 0};
    bool triclinic = false;
    bool bounds_changed = false;
    double domain_ghost_cutoff = 0.0;
    // BoundaryType per axis (domain.rs:36-44): 0 periodic, 1 fixed, 2 shrink-wrap
    int btype[3] = {0, 0, 0};
    double shrink_wrap_padding = 0.0;
    bool is_periodic(int d) const { return btype[d] == 0; }

    // ---- Neighbor (neighbor.rs:87-174) ----
    double skin_fraction = 1.0, bin_min_size = 1.0, additive_skin = 0.0;
    uint64_t every = 0, sort_every = 1000;
    bool check = true, newton = true;
    std::vector<uint32_t> neighbor_offsets, neighbor_indices;
    V3 bin_size{1, 1, 1};
    int32_t bin_count[3] = {1, 1, 1};
    std::vector<V3> last_build_pos;
    size_t steps_since_build = 0, last_build_total = 0;
    V3 pbc_box{0, 0, 0};
    bool pbc_flags[3] = {true, true, true};
    std::vector<int32_t> bin_stencil, bin_stencil_forward;
    bool bin_stencil_self = false;
    V3 bin_origin{0, 0, 0};
    size_t bin_total_cells = 0;
    double ghost_cutoff = 0.0;
    double cached_min_skin = DBL_MAX;
    size_t sort_counter = 0;
    std::vector<uint32_t> sorted_local_cell;
    bool local_cells_valid = false;
    bool has_uniform_cutoff = false;
    double uniform_cutoff_sq = 0.0;
    double cached_max_cutoff = 0.0;

    // ---- CommTopology (comm.rs:127-133), single rank: rank 0, grid 1x1x1 ----
    int swap_directions[2][3] = {{-1, -1, -1}, {-1, -1, -1}};
    double periodic_swap[2][3] = {{0, 0, 0}, {0, 0, 0}};
    std::vector<Swap> swaps;
    int maxneed[3] = {0, 0, 0};

    State state = FULL_REBUILD;

    // ---- DeformState (soil_deform/src/lib.rs:195-211) ----
    // per-axis style (AxisDeform, lib.rs:168-190): 0 none, 1 erate (a = rate),
    // 2 vel (a = velocity), 3 final (a, b = target lo, hi; stage = the run
    // stage's total steps, RunState cycle_count + cycle_remaining)
    struct Axis {
        int style = 0;
        double a = 0.0, b = 0.0;
        uint64_t stage = 0;
        double lo_0 = 0.0, hi_0 = 0.0;
    } axes[3];
    bool remap = true;
    bool shear = false;
    double shear_rate = 0.0;
    bool shear_initialized = false;
    bool deform_initialized = false;
    size_t deform_step = 0;

    // ---- built-in consumer ----
    double harmonic_k = 0.0;
    int radius_col = -1;

    // ---- bookkeeping ----
    bool setup_done = false;
    uint64_t steps_done = 0, rebuilds = 0, sorts = 0;
    std::vector<size_t> last_perm;

    size_t len() const { return pos.size(); }

    // Domain::x2lamda, domain.rs:211-217
    V3 x2lamda(const V3& r) const {
        double xy = tilt[0], xz = tilt[1], yz = tilt[2];
        double lz = (r[2] - blo[2]) / size[2];
        double ly = (r[1] - blo[1] - yz * lz) / size[1];
        double lx = (r[0] - blo[0] - xy * ly - xz * lz) / size[0];
        return {lx, ly, lz};
    }
    // Domain::lamda2x, domain.rs:222-229
    V3 lamda2x(const V3& l) const {
        double xy = tilt[0], xz = tilt[1], yz = tilt[2];
        return {blo[0] + size[0] * l[0] + xy * l[1] + xz * l[2],
                blo[1] + size[1] * l[1] + yz * l[2],
                blo[2] + size[2] * l[2]};
    }

    // ---------------------------------------------------------------------
    // Atom structural ops
    // ---------------------------------------------------------------------
    void push_atom(uint32_t t, uint32_t ty, int32_t orig, const V3& p, const V3& v, const V3& f,
                   double cut, double m, double im, const I3& img, bool ghost) {
        tag.push_back(t);
        atom_type.push_back(ty);
        origin_index.push_back(orig);
        pos.push_back(p);
        vel.push_back(v);
        force.push_back(f);
        cutoff_radius.push_back(cut);
        mass.push_back(m);
        inv_mass.push_back(im);
        image.push_back(img);
        is_ghost.push_back(ghost ? 1 : 0);
    }
    // Atom::truncate_to_nlocal + AtomDataRegistry::truncate_all (atom.rs:465-472, 261-266)
    void truncate_to(size_t n) {
        tag.resize(n); atom_type.resize(n); origin_index.resize(n); is_ghost.resize(n);
        pos.resize(n); vel.resize(n); force.resize(n); cutoff_radius.resize(n);
        mass.resize(n); inv_mass.resize(n); image.resize(n);
        for (auto& c : cols) c.data.resize(n * (size_t)c.width);
    }
    // Atom::apply_permutation (atom.rs:479-490) + registry (atom.rs:284-289)
    template <class T>
    static void permute_vec(std::vector<T>& v, const std::vector<size_t>& perm, size_t n) {
        std::vector<T> s(perm.size());
        for (size_t k = 0; k < perm.size(); ++k) s[k] = v[perm[k]];
        for (size_t k = 0; k < n; ++k) v[k] = s[k];
    }
    void apply_permutation(const std::vector<size_t>& perm, size_t n) {
        permute_vec(tag, perm, n); permute_vec(atom_type, perm, n);
        permute_vec(origin_index, perm, n); permute_vec(is_ghost, perm, n);
        permute_vec(pos, perm, n); permute_vec(vel, perm, n); permute_vec(force, perm, n);
        permute_vec(cutoff_radius, perm, n); permute_vec(mass, perm, n);
        permute_vec(inv_mass, perm, n); permute_vec(image, perm, n);
        for (auto& c : cols) {  // derive apply_permutation: per field, gather then copy
            std::vector<double> s(perm.size() * (size_t)c.width);
            for (size_t k = 0; k < perm.size(); ++k)
                for (int w = 0; w < c.width; ++w) s[k * c.width + w] = c.data[perm[k] * c.width + w];
            for (size_t k = 0; k < n * (size_t)c.width; ++k) c.data[k] = s[k];
        }
    }

    // ---------------------------------------------------------------------
    // Setup
    // ---------------------------------------------------------------------
    // comm_setup, comm.rs:253-283 (rank 0 of a 1x1x1 grid, all axes periodic)
    // comm_setup, comm.rs:253-283 (grid 1x1x1): a periodic axis sends to
    // itself with a shift, a non-periodic one has no neighbor (-1)
    void comm_setup() {
        for (int dim = 0; dim < 3; ++dim) {
            if (is_periodic(dim)) {
                swap_directions[1][dim] = 0;
                periodic_swap[1][dim] = -1.0;
                swap_directions[0][dim] = 0;
                periodic_swap[0][dim] = 1.0;
            } else {
                swap_directions[0][dim] = swap_directions[1][dim] = -1;
                periodic_swap[0][dim] = periodic_swap[1][dim] = 0.0;
            }
        }
    }

    // compute_bin_grid, neighbor.rs:311-397 (comm_size = 1)
    void compute_bin_grid() {
        double max_cutoff = cached_max_cutoff;
        double required_bin = max_cutoff;
        double min_bin = std::max(bin_min_size, required_bin);
        if (triclinic) {
            compute_bin_grid_triclinic(max_cutoff, min_bin);
            return;
        }
        int32_t xi = sat_i32(std::max(std::floor(sub_len[0] / min_bin), 1.0));
        int32_t yi = sat_i32(std::max(std::floor(sub_len[1] / min_bin), 1.0));
        int32_t zi = sat_i32(std::max(std::floor(sub_len[2] / min_bin), 1.0));
        V3 abs_{sub_len[0] / (double)xi, sub_len[1] / (double)yi, sub_len[2] / (double)zi};
        double ghost_cut = domain_ghost_cutoff > max_cutoff ? domain_ghost_cutoff : max_cutoff;
        int32_t srx = sat_i32(std::ceil(max_cutoff / abs_[0]));
        int32_t sry = sat_i32(std::ceil(max_cutoff / abs_[1]));
        int32_t srz = sat_i32(std::ceil(max_cutoff / abs_[2]));
        int32_t sx = sat_i32(std::ceil(ghost_cut / abs_[0])) + srx;
        int32_t sy = sat_i32(std::ceil(ghost_cut / abs_[1])) + sry;
        int32_t sz = sat_i32(std::ceil(ghost_cut / abs_[2])) + srz;
        int32_t nx = xi + 2 * sx, ny = yi + 2 * sy, nz = zi + 2 * sz;
        bin_count[0] = nx; bin_count[1] = ny; bin_count[2] = nz;
        bin_size = abs_;
        bin_total_cells = (size_t)(nx * ny * nz);
        bin_origin = {sub_lo[0] - abs_[0] * (double)sx, sub_lo[1] - abs_[1] * (double)sy,
                      sub_lo[2] - abs_[2] * (double)sz};
        double cutoff_sq = max_cutoff * max_cutoff;
        bin_stencil.clear();
        bin_stencil_forward.clear();
        bin_stencil_self = false;
        for (int32_t dx = -sx; dx <= sx; ++dx)
            for (int32_t dy = -sy; dy <= sy; ++dy)
                for (int32_t dz = -sz; dz <= sz; ++dz) {
                    double mdx = (double)(std::abs(dx) > 0 ? std::abs(dx) - 1 : 0) * abs_[0];
                    double mdy = (double)(std::abs(dy) > 0 ? std::abs(dy) - 1 : 0) * abs_[1];
                    double mdz = (double)(std::abs(dz) > 0 ? std::abs(dz) - 1 : 0) * abs_[2];
                    if (mdx * mdx + mdy * mdy + mdz * mdz < cutoff_sq) {
                        int32_t off = dx * ny * nz + dy * nz + dz;
                        bin_stencil.push_back(off);
                        if (off > 0) bin_stencil_forward.push_back(off);
                        else if (off == 0) bin_stencil_self = true;
                    }
                }
        pbc_box = {bhi[0] - blo[0], bhi[1] - blo[1], bhi[2] - blo[2]};
    }

    // compute_bin_grid_triclinic, neighbor.rs:411-495
    void compute_bin_grid_triclinic(double max_cutoff, double min_bin) {
        V3 l = size;
        double xy = tilt[0];
        V3 sub_l{sub_lam_hi[0] - sub_lam_lo[0], sub_lam_hi[1] - sub_lam_lo[1],
                 sub_lam_hi[2] - sub_lam_lo[2]};
        int32_t ni[3];
        for (int d = 0; d < 3; ++d) ni[d] = sat_i32(std::max(std::floor(sub_l[d] * l[d] / min_bin), 1.0));
        V3 bl{sub_l[0] / (double)ni[0], sub_l[1] / (double)ni[1], sub_l[2] / (double)ni[2]};
        V3 real_bin{bl[0] * l[0], bl[1] * l[1], bl[2] * l[2]};
        double ghost_cut = domain_ghost_cutoff > max_cutoff ? domain_ghost_cutoff : max_cutoff;
        int32_t sr[3];
        for (int d = 0; d < 3; ++d) sr[d] = sat_i32(std::ceil(max_cutoff / real_bin[d]));
        int32_t skew_x_bins = sat_i32(std::ceil(std::fabs(xy) / real_bin[0]));
        int32_t sx = sat_i32(std::ceil(ghost_cut / real_bin[0])) + sr[0] + skew_x_bins;
        int32_t sy = sat_i32(std::ceil(ghost_cut / real_bin[1])) + sr[1];
        int32_t sz = sat_i32(std::ceil(ghost_cut / real_bin[2])) + sr[2];
        int32_t nx = ni[0] + 2 * sx, ny = ni[1] + 2 * sy, nz = ni[2] + 2 * sz;
        bin_count[0] = nx; bin_count[1] = ny; bin_count[2] = nz;
        bin_size = bl;
        bin_total_cells = (size_t)(nx * ny * nz);
        bin_origin = {sub_lam_lo[0] - bl[0] * (double)sx, sub_lam_lo[1] - bl[1] * (double)sy,
                      sub_lam_lo[2] - bl[2] * (double)sz};
        double cutoff_sq = max_cutoff * max_cutoff;
        bin_stencil.clear();
        bin_stencil_forward.clear();
        bin_stencil_self = false;
        for (int32_t dx = -sx; dx <= sx; ++dx)
            for (int32_t dy = -sy; dy <= sy; ++dy)
                for (int32_t dz = -sz; dz <= sz; ++dz) {
                    double m1 = (double)(std::abs(dy) > 0 ? std::abs(dy) - 1 : 0) * bl[1];
                    double m2 = (double)(std::abs(dz) > 0 ? std::abs(dz) - 1 : 0) * bl[2];
                    double dyz_sq = (l[1] * m1) * (l[1] * m1) + (l[2] * m2) * (l[2] * m2);
                    if (dyz_sq >= cutoff_sq) continue;
                    double budget = std::sqrt(cutoff_sq - dyz_sq);
                    double a_lo = l[0] * ((double)dx - 1.0) * bl[0];
                    double a_hi = l[0] * ((double)dx + 1.0) * bl[0];
                    double b1 = xy * ((double)dy - 1.0) * bl[1];
                    double b2 = xy * ((double)dy + 1.0) * bl[1];
                    double b_lo = b1 <= b2 ? b1 : b2;
                    double b_hi = b1 <= b2 ? b2 : b1;
                    double lo = a_lo + b_lo;
                    double hi = a_hi + b_hi;
                    if (hi >= -budget && lo <= budget) {
                        int32_t off = dx * ny * nz + dy * nz + dz;
                        bin_stencil.push_back(off);
                        if (off > 0) bin_stencil_forward.push_back(off);
                        else if (off == 0) bin_stencil_self = true;
                    }
                }
        pbc_box = l;
    }

    // neighbor_setup, neighbor.rs:604-665 (comm_size = 1)
    void neighbor_setup() {
        double local_max_skin = 0.0;
        for (double c : cutoff_radius) local_max_skin = std::max(local_max_skin, c);
        double max_skin = local_max_skin;
        double max_cutoff = max_skin > 0.0 ? 2.0 * max_skin * skin_fraction : bin_min_size;
        double min_skin = DBL_MAX;
        for (double c : cutoff_radius) min_skin = std::min(min_skin, c);
        double displacement_buffer = 0.0;
        if (min_skin < DBL_MAX * 0.5) {
            displacement_buffer = (skin_fraction - 1.0) * min_skin;
            if (additive_skin != 0.0) displacement_buffer = displacement_buffer + 0.5 * additive_skin;
        }
        double ghost_cut = std::max(max_cutoff + 2.0 * displacement_buffer, domain_ghost_cutoff);
        ghost_cutoff = ghost_cut;
        cached_max_cutoff = max_cutoff;
        domain_ghost_cutoff = ghost_cut;
        double required_bin = max_cutoff;
        if (bin_min_size < required_bin) bin_min_size = required_bin;
        compute_bin_grid();
        for (int d = 0; d < 3; ++d) pbc_flags[d] = is_periodic(d);  // neighbor.rs:656
    }

    // setup_deform, soil_deform/src/lib.rs:346-420
    void setup_deform() {
        shear_initialized = false;
        for (int d = 0; d < 3; ++d)
            if (axes[d].style) {
                axes[d].lo_0 = blo[d];
                axes[d].hi_0 = bhi[d];
            }
        deform_initialized = true;
        deform_step = 0;
    }

    // ---------------------------------------------------------------------
    // Per-step systems
    // ---------------------------------------------------------------------
    // apply_deform, soil_deform/src/lib.rs:435-604: orthogonal axes (lib.rs:
    // 468-557), then the xy shear.  Returns false when an axis collapses (the
    // reference panics).
    bool phase_deform() {
        if (!deform_initialized || !(shear || axes[0].style || axes[1].style || axes[2].style))
            return true;
        deform_step += 1;
        size_t nl = nlocal;
        bool box_changed = false;
        for (int dim = 0; dim < 3; ++dim) {
            const Axis& ax = axes[dim];
            if (!ax.style) continue;
            double old_lo = blo[dim], old_hi = bhi[dim];
            double old_size = old_hi - old_lo;
            double l0 = ax.hi_0 - ax.lo_0;
            double new_lo, new_hi;
            if (ax.style == 1) {
                double scale = 1.0 + ax.a * dt * (double)deform_step;
                double new_l = l0 * scale;
                double center = (ax.lo_0 + ax.hi_0) * 0.5;
                new_lo = center - new_l * 0.5;
                new_hi = center + new_l * 0.5;
            } else if (ax.style == 2) {
                double delta = ax.a * dt * (double)deform_step;
                double new_l = l0 + delta;
                double center = (ax.lo_0 + ax.hi_0) * 0.5;
                new_lo = center - new_l * 0.5;
                new_hi = center + new_l * 0.5;
            } else {
                double frac = ax.stage > 0 ? (double)deform_step / (double)ax.stage : 1.0;
                frac = std::min(frac, 1.0);
                new_lo = ax.lo_0 + (ax.a - ax.lo_0) * frac;
                new_hi = ax.hi_0 + (ax.b - ax.hi_0) * frac;
            }
            double new_size = new_hi - new_lo;
            if (new_size <= 0.0) return false;
            if (remap && old_size > 0.0) {
                double scale = new_size / old_size;
                double new_center = (new_lo + new_hi) * 0.5;
                double old_center = (old_lo + old_hi) * 0.5;
                for (size_t i = 0; i < nl; ++i)
                    pos[i][dim] = new_center + (pos[i][dim] - old_center) * scale;
            }
            blo[dim] = new_lo;
            bhi[dim] = new_hi;
            size[dim] = new_size;
            sub_lo[dim] = new_lo;
            sub_hi[dim] = new_hi;
            sub_len[dim] = new_size;
            box_changed = true;
        }
        if (box_changed) {
            bounds_changed = true;
            last_build_pos.clear();
        }
        if (!shear) return true;
        double rate = shear_rate;
        double lx = size[0], ly = size[1];
        double dv = rate * ly;
        if (!shear_initialized) {
            double yc = 0.5 * (blo[1] + bhi[1]);
            for (size_t i = 0; i < nl; ++i) vel[i][0] += rate * (pos[i][1] - yc);
            shear_initialized = true;
        }
        double raw = rate * dt * (double)deform_step * ly;
        double xy = raw - lx * rround(raw / lx);
        tilt[0] = xy;
        bvel[0] = dv;
        triclinic = true;
        bounds_changed = true;
        last_build_pos.clear();  // box_changed: force a rebuild (lib.rs:590-603)
        return true;
    }

    // initial_integration, soil_verlet/src/lib.rs:131-162
    void phase_initial() {
        double dt_a = dt;
        for (size_t i = 0; i < nlocal; ++i) {
            double h = 0.5 * dt_a * inv_mass[i];
            const V3& f = force[i];
            V3& v = vel[i];
            double v0 = v[0] + h * f[0];
            double v1 = v[1] + h * f[1];
            double v2 = v[2] + h * f[2];
            v[0] = v0; v[1] = v1; v[2] = v2;
            V3& p = pos[i];
            p[0] = p[0] + v0 * dt_a;
            p[1] = p[1] + v1 * dt_a;
            p[2] = p[2] + v2 * dt_a;
        }
    }

    // final_integration, soil_verlet/src/lib.rs:175-194
    void phase_final() {
        double dt_a = dt;
        for (size_t i = 0; i < nlocal; ++i) {
            double h = 0.5 * dt_a * inv_mass[i];
            const V3& f = force[i];
            V3& v = vel[i];
            v[0] = v[0] + h * f[0];
            v[1] = v[1] + h * f[1];
            v[2] = v[2] + h * f[2];
        }
    }

    // displacement_exceeded, neighbor.rs:693-758 (fully periodic fast path;
    // the box is always periodic on all axes here)
    bool displacement_exceeded() const {
        double min_r = cached_min_skin;
        double per_atom_skin = (skin_fraction - 1.0) * min_r;
        if (additive_skin != 0.0) per_atom_skin = per_atom_skin + 0.5 * additive_skin;
        double threshold_sq = per_atom_skin * per_atom_skin;
        double bx = pbc_box[0], by = pbc_box[1], bz = pbc_box[2];
        size_t n = last_build_pos.size();
        if (!(pbc_flags[0] && pbc_flags[1] && pbc_flags[2])) {
            // general path, neighbor.rs:736-756: per-axis single-image correction
            double hbx = bx * 0.5, hby = by * 0.5, hbz = bz * 0.5;
            for (size_t idx = 0; idx < n; ++idx) {
                double dx = pos[idx][0] - last_build_pos[idx][0];
                double dy = pos[idx][1] - last_build_pos[idx][1];
                double dz = pos[idx][2] - last_build_pos[idx][2];
                if (pbc_flags[0]) { if (dx > hbx) dx -= bx; else if (dx < -hbx) dx += bx; }
                if (pbc_flags[1]) { if (dy > hby) dy -= by; else if (dy < -hby) dy += by; }
                if (pbc_flags[2]) { if (dz > hbz) dz -= bz; else if (dz < -hbz) dz += bz; }
                if (dx * dx + dy * dy + dz * dz > threshold_sq) return true;
            }
            return false;
        }
        double ibx = 1.0 / bx, iby = 1.0 / by, ibz = 1.0 / bz;
        for (size_t idx = 0; idx < n; ++idx) {
            const V3& p = pos[idx];
            const V3& q = last_build_pos[idx];
            double dx = p[0] - q[0], dy = p[1] - q[1], dz = p[2] - q[2];
            dx -= bx * rround(dx * ibx);
            dy -= by * rround(dy * iby);
            dz -= bz * rround(dz * ibz);
            if (std::fma(dx, dx, std::fma(dy, dy, dz * dz)) > threshold_sq) return true;
        }
        return false;
    }

    // needs_rebuild, neighbor.rs:762-784
    bool needs_rebuild() const {
        size_t nl = nlocal;
        if (last_build_pos.size() != nl || nl == 0) return true;
        if (state == FULL_REBUILD) return true;
        if (every == 0) return displacement_exceeded();
        if (check) return steps_since_build >= every || displacement_exceeded();
        return steps_since_build >= every;
    }

    // decide_rebuild, neighbor.rs:796-822 (run_if CommunicateOnly)
    void phase_decide_rebuild() {
        if (state != COMMUNICATE_ONLY) return;
        if (needs_rebuild()) state = FULL_REBUILD;
        else steps_since_build += 1;
    }

    // remove_ghost_atoms, atom.rs:625-629 (run_if FullRebuild)
    void phase_remove_ghosts() {
        if (state != FULL_REBUILD) return;
        truncate_to(nlocal);
        nghost = 0;
    }

    // zero_all_forces, atom.rs:631-635 (+ derive zero(), soil_derive/src/lib.rs:468-500)
    void phase_zero_forces() {
        size_t n = len();
        for (size_t i = 0; i < n; ++i) force[i] = {0.0, 0.0, 0.0};
        for (auto& c : cols)
            if (c.flags & SOIL_COL_ZERO) {
                c.data.resize(n * (size_t)c.width, 0.0);
                std::fill(c.data.begin(), c.data.begin() + n * (size_t)c.width, 0.0);
            }
    }

    // wrap_periodic, domain.rs:594-605
    static double wrap_periodic(double p, double low, double sz, int32_t* delta) {
        double high = low + sz;
        if (p < low) { *delta = -1; return p + sz; }
        if (p >= high) { *delta = 1; return p - sz; }
        *delta = 0;
        return p;
    }

    // pbc, domain.rs:611-663 (fully periodic fast path) / pbc_triclinic 674-729
    void phase_pbc() {
        if (state != FULL_REBUILD) return;
        if (triclinic) {  // pbc_triclinic, domain.rs:673-729
            size_t removed = 0;
            for (size_t ii = nlocal; ii-- > 0;) {
                V3 lam = x2lamda(pos[ii]);
                int32_t delta[3] = {0, 0, 0};
                bool gone = false;
                for (int d = 0; d < 3 && !gone; ++d) {
                    if (is_periodic(d)) {
                        if (lam[d] < 0.0) { lam[d] += 1.0; delta[d] = -1; }
                        else if (lam[d] >= 1.0) { lam[d] -= 1.0; delta[d] = 1; }
                    } else if (lam[d] < 0.0 || lam[d] >= 1.0) {
                        swap_remove(ii);
                        removed += 1;
                        gone = true;
                    }
                }
                if (gone) continue;
                pos[ii] = lamda2x(lam);
                for (int d = 0; d < 3; ++d) image[ii][d] += delta[d];
                if (delta[1] != 0) {
                    double s = (double)delta[1];
                    vel[ii][0] -= s * bvel[0];
                    vel[ii][1] -= s * bvel[1];
                    vel[ii][2] -= s * bvel[2];
                }
            }
            if (removed > 0) {
                nlocal = (uint32_t)(nlocal - removed);
                state = FULL_REBUILD;
            }
            return;
        }
        if (is_periodic(0) && is_periodic(1) && is_periodic(2)) {
            for (size_t i = 0; i < nlocal; ++i)
                for (int d = 0; d < 3; ++d) {
                    int32_t delta;
                    pos[i][d] = wrap_periodic(pos[i][d], blo[d], size[d], &delta);
                    image[i][d] += delta;
                }
            return;
        }
        // slow path (domain.rs:641-662): wrap periodic axes; remove atoms
        // outside a non-periodic axis by swap_remove, last index first
        size_t removed = 0;
        for (size_t i = nlocal; i-- > 0;) {
            for (int d = 0; d < 3; ++d) {
                if (is_periodic(d)) {
                    int32_t delta;
                    pos[i][d] = wrap_periodic(pos[i][d], blo[d], size[d], &delta);
                    image[i][d] += delta;
                } else if (pos[i][d] < blo[d] || pos[i][d] >= bhi[d]) {
                    swap_remove(i);
                    removed += 1;
                    break;
                }
            }
        }
        if (removed > 0) {
            nlocal = (uint32_t)(nlocal - removed);
            state = FULL_REBUILD;
        }
    }

    // Atom::swap_remove (atom.rs:456-458) + registry swap_remove_all (268-272)
    template <class T>
    static void swap_remove_vec(std::vector<T>& v, size_t i) {
        v[i] = v.back();
        v.pop_back();
    }
    void swap_remove(size_t i) {
        swap_remove_vec(tag, i); swap_remove_vec(atom_type, i); swap_remove_vec(origin_index, i);
        swap_remove_vec(is_ghost, i); swap_remove_vec(pos, i); swap_remove_vec(vel, i);
        swap_remove_vec(force, i); swap_remove_vec(cutoff_radius, i); swap_remove_vec(mass, i);
        swap_remove_vec(inv_mass, i); swap_remove_vec(image, i);
        for (auto& c : cols) {
            const size_t w = (size_t)c.width, last = c.data.size() / w - 1;
            for (size_t k = 0; k < w; ++k) c.data[i * w + k] = c.data[last * w + k];
            c.data.resize(last * w);
        }
    }

    // shrink_wrap_update, domain.rs:509-575 (every step, before pbc)
    void phase_shrink_wrap() {
        bool any = btype[0] == 2 || btype[1] == 2 || btype[2] == 2;
        size_t nl = nlocal;
        if (!any || nl == 0) return;
        double padding;
        if (shrink_wrap_padding > 0.0) padding = shrink_wrap_padding;
        else if (domain_ghost_cutoff > 0.0) padding = domain_ghost_cutoff;
        else {
            double mx = std::max(size[0], std::max(size[1], size[2]));
            padding = mx > 0.0 ? mx * 0.01 : 1.0;
        }
        bool changed = false;
        for (int d = 0; d < 3; ++d) {
            if (btype[d] != 2) continue;
            double mn = DBL_MAX, mxp = -DBL_MAX;
            for (size_t i = 0; i < nl; ++i) {
                double p = pos[i][d];
                if (p < mn) mn = p;
                if (p > mxp) mxp = p;
            }
            double new_low = mn - padding, new_high = mxp + padding;
            const double tol = 1e-12;
            if (std::fabs(new_low - blo[d]) > tol || std::fabs(new_high - bhi[d]) > tol) {
                blo[d] = new_low;
                bhi[d] = new_high;
                sub_lo[d] = new_low;
                sub_hi[d] = new_high;
                changed = true;
            }
        }
        if (changed) {  // update_derived, domain.rs:171-177
            for (int d = 0; d < 3; ++d) {
                size[d] = bhi[d] - blo[d];
                sub_len[d] = sub_hi[d] - sub_lo[d];
            }
            bounds_changed = true;
        }
    }

    // cell of a position for the current grid (sort_atoms_by_bin 912-923,
    // bin_neighbor_list 1070-1083: identical formula)
    uint32_t cell_of(const V3& pr) const {
        V3 p = triclinic ? x2lamda(pr) : pr;
        double inv_bsx = 1.0 / bin_size[0], inv_bsy = 1.0 / bin_size[1], inv_bsz = 1.0 / bin_size[2];
        int32_t nx = bin_count[0], ny = bin_count[1], nz = bin_count[2];
        int32_t cx = clampi(sat_i32(std::floor((p[0] - bin_origin[0]) * inv_bsx)), 0, nx - 1);
        int32_t cy = clampi(sat_i32(std::floor((p[1] - bin_origin[1]) * inv_bsy)), 0, ny - 1);
        int32_t cz = clampi(sat_i32(std::floor((p[2] - bin_origin[2]) * inv_bsz)), 0, nz - 1);
        return (uint32_t)(cx * ny * nz + cy * nz + cz);
    }

    // sort_atoms_by_bin, neighbor.rs:834-997
    void phase_sort() {
        if (bounds_changed) {
            if (cached_max_cutoff > 0.0) compute_bin_grid();  // recompute_bins 498-503
            bounds_changed = false;
            state = FULL_REBUILD;
        }
        sort_counter += 1;
        bool periodic_sort = sort_every > 0 && sort_counter >= sort_every;
        if (periodic_sort) sort_counter = 0;
        size_t nl = nlocal;
        local_cells_valid = false;
        if (nl == 0 || bin_total_cells == 0 || nl > pos.size()) return;
        bool full_rebuild = state == FULL_REBUILD;
        if (!periodic_sort && !full_rebuild) return;

        size_t total_cells = bin_total_cells;
        std::vector<uint32_t> cell(nl);
        std::vector<uint32_t> counts(total_cells + 1, 0);
        std::vector<size_t> perm(nl);
        for (size_t i = 0; i < nl; ++i) {
            uint32_t c = cell_of(pos[i]);
            cell[i] = c;
            counts[(size_t)c + 1] += 1;
        }
        for (size_t c = 0; c < total_cells; ++c) counts[c + 1] += counts[c];
        for (size_t i = 0; i < nl; ++i) {
            uint32_t c = cell[i];
            uint32_t slot = counts[c];
            perm[slot] = i;
            counts[c] = slot + 1;
        }
        bool already_sorted = true;
        for (size_t i = 0; i < nl; ++i)
            if (perm[i] != i) { already_sorted = false; break; }
        sorted_local_cell.assign(nl, 0);
        for (size_t k = 0; k < nl; ++k) sorted_local_cell[k] = cell[perm[k]];
        local_cells_valid = true;
        sorts += 1;
        last_perm = perm;
        if (!already_sorted) {
            apply_permutation(perm, nl);
            if (last_build_pos.size() >= nl) {
                std::vector<V3> scratch(last_build_pos.begin(), last_build_pos.begin() + nl);
                for (size_t k = 0; k < nl; ++k) last_build_pos[k] = scratch[perm[k]];
            }
        }
        if (periodic_sort && !already_sorted) {
            last_build_pos.clear();
            state = FULL_REBUILD;
        }
    }

    // pack_border_atoms, comm.rs:288-358 (ghost_cutoff > 0 always here)
    void pack_border_atoms(int dim, int swap, const V3& change_pos, const V3& vel_offset,
                           std::vector<size_t>& packed, size_t scan_end, double gc,
                           bool self_send) {
        packed.clear();
        if (triclinic) {
            double lo_face = sub_lam_lo[dim], hi_face = sub_lam_hi[dim];
            double inflate = dim == 0 ? 1.0 + std::fabs(tilt[0]) / size[1] : 1.0;
            double cut_l = (gc / size[dim]) * inflate;
            for (size_t i = 0; i < scan_end; ++i) {
                double lam = x2lamda(pos[i])[dim];
                bool in_skin = swap == 0 ? lam < lo_face + cut_l : lam >= hi_face - cut_l;
                if (in_skin) packed.push_back(i);
            }
        } else {
            double lo_face = sub_lo[dim], hi_face = sub_hi[dim];
            double thresh = swap == 0 ? lo_face + gc : hi_face - gc;
            for (size_t i = 0; i < scan_end; ++i) {
                double p = pos[i][dim];
                bool in_skin = swap == 0 ? p < thresh : p >= thresh;
                if (in_skin) packed.push_back(i);
            }
        }
        // self-send: pack_border (atom.rs:520-539 layout) then unpack_atom (539-553)
        // and registry pack_all/unpack_all; appended in scan order.  Without a
        // neighbor (non-periodic axis, comm.rs:832-835) the packed atoms go nowhere.
        if (!self_send) return;
        std::vector<size_t> src = packed;
        for (size_t i : src) {
            V3 p{pos[i][0] + change_pos[0], pos[i][1] + change_pos[1], pos[i][2] + change_pos[2]};
            V3 v{vel[i][0] + vel_offset[0], vel[i][1] + vel_offset[1], vel[i][2] + vel_offset[2]};
            V3 f = force[i];
            I3 img = image[i];
            double m = mass[i];
            push_atom(tag[i], atom_type[i], (int32_t)i, p, v, f, cutoff_radius[i], m, 1.0 / m, img, true);
            for (auto& c : cols)
                for (int w = 0; w < c.width; ++w) {
                    double val = c.data[i * c.width + w];
                    c.data.push_back(val);
                }
            nghost += 1;
        }
    }

    // borders, comm.rs:682-860 (single rank: every swap is a self-send)
    void phase_borders() {
        if (state != FULL_REBUILD) return;
        if (nghost > 0) {
            truncate_to(nlocal);
            nghost = 0;
        }
        nlocal = (uint32_t)len();
        nghost = 0;
        if (maxneed[0] == 0 && maxneed[1] == 0 && maxneed[2] == 0)
            maxneed[0] = maxneed[1] = maxneed[2] = 1;  // decomp[dim] == 1
        size_t swap_idx = 0;
        size_t scan_end = nlocal;
        for (int dim = 0; dim < 3; ++dim) {
            for (int need = 0; need < maxneed[dim]; ++need) {
                size_t dim_scan_end = scan_end;
                for (int swap = 0; swap < 2; ++swap) {
                    int to_proc = swap_directions[swap][dim];
                    int from_proc = swap_directions[(swap + 1) % 2][dim];
                    double po = periodic_swap[swap][dim];
                    V3 pbc_shift;
                    if (dim == 0) pbc_shift = {po * size[0], 0.0, 0.0};
                    else if (dim == 1) pbc_shift = {po * tilt[0], po * size[1], 0.0};
                    else pbc_shift = {po * tilt[1], po * tilt[2], po * size[2]};
                    V3 vel_shift = dim == 1 ? V3{po * bvel[0], po * bvel[1], po * bvel[2]} : V3{0.0, 0.0, 0.0};
                    if (swap_idx == swaps.size()) swaps.emplace_back();
                    Swap& e = swaps[swap_idx];
                    size_t recv_start = len();
                    const bool self_send = to_proc == 0;
                    pack_border_atoms(dim, swap, pbc_shift, vel_shift, e.send_indices, dim_scan_end,
                                      domain_ghost_cutoff, self_send);
                    e.recv_start = recv_start;
                    e.recv_count = self_send ? e.send_indices.size() : 0;
                    e.to_proc = to_proc;
                    e.from_proc = from_proc;
                    e.periodic_offset = pbc_shift;
                    e.vel_offset = vel_shift;
                    swap_idx += 1;
                }
                scan_end = (size_t)nlocal + nghost;
            }
        }
        swaps.resize(swap_idx);
    }

    // forward_comm self-send path, comm.rs:400-432, 439-470, 496-573
    void phase_forward_comm() {
        if (state != COMMUNICATE_ONLY) return;
        for (const Swap& s : swaps) {
            if (s.to_proc < 0 || s.from_proc < 0) continue;  // no neighbor (comm.rs:460)
            // pack then unpack (forward_prepare_swap), swaps in recorded order
            size_t n = s.send_indices.size();
            std::vector<double> buf;
            buf.reserve(n * 6);
            for (size_t idx : s.send_indices) {
                for (int d = 0; d < 3; ++d) buf.push_back(pos[idx][d] + s.periodic_offset[d]);
                for (int d = 0; d < 3; ++d) buf.push_back(vel[idx][d] + s.vel_offset[d]);
            }
            std::vector<double> fbuf;
            for (size_t idx : s.send_indices)
                for (auto& c : cols)
                    if (c.flags & SOIL_COL_FORWARD)
                        for (int w = 0; w < c.width; ++w) fbuf.push_back(c.data[idx * c.width + w]);
            size_t fw = n ? fbuf.size() / n : 0;
            for (size_t k = 0; k < s.recv_count; ++k) {
                size_t g = s.recv_start + k;
                pos[g] = {buf[k * 6 + 0], buf[k * 6 + 1], buf[k * 6 + 2]};
                vel[g] = {buf[k * 6 + 3], buf[k * 6 + 4], buf[k * 6 + 5]};
                size_t o = 0;
                for (auto& c : cols)
                    if (c.flags & SOIL_COL_FORWARD)
                        for (int w = 0; w < c.width; ++w) c.data[g * c.width + w] = fbuf[k * fw + o++];
            }
        }
    }

    // save_build_positions, neighbor.rs:669-690
    void save_build_positions() {
        size_t nl = nlocal;
        last_build_pos.assign(pos.begin(), pos.begin() + nl);
        last_build_total = len();
        steps_since_build = 0;
        double mn = DBL_MAX, mx = -DBL_MAX;
        for (size_t i = 0; i < nl; ++i) {
            mn = std::min(mn, cutoff_radius[i]);
            mx = std::max(mx, cutoff_radius[i]);
        }
        cached_min_skin = mn;
        if (std::fabs(mx - mn) < 1e-15) {
            double cutoff = 2.0 * mn * skin_fraction;
            has_uniform_cutoff = true;
            uniform_cutoff_sq = cutoff * cutoff;
        } else {
            has_uniform_cutoff = false;
        }
    }

    // bin_neighbor_list, neighbor.rs:1013-1319
    void phase_neighbor() {
        if (state != FULL_REBUILD) return;
        size_t nl = nlocal, total = len();
        state = COMMUNICATE_ONLY;
        save_build_positions();
        size_t total_cells = bin_total_cells;
        std::vector<uint32_t> atom_cell(total, 0);
        std::vector<uint32_t> cnt(total_cells, 0);
        bool reuse_local = local_cells_valid && sorted_local_cell.size() == nl;
        size_t ghost_start = 0;
        if (reuse_local) {
            for (size_t i = 0; i < nl; ++i) {
                atom_cell[i] = sorted_local_cell[i];
                cnt[sorted_local_cell[i]] += 1;
            }
            ghost_start = nl;
        }
        for (size_t i = ghost_start; i < total; ++i) {
            uint32_t c = cell_of(pos[i]);
            atom_cell[i] = c;
            cnt[c] += 1;
        }
        local_cells_valid = false;
        std::vector<uint32_t> bin_start(total_cells + 1, 0);
        for (size_t c = 0; c < total_cells; ++c) bin_start[c + 1] = bin_start[c] + cnt[c];
        std::vector<uint32_t> sorted_atoms(total), atom_sorted_idx(total);
        for (size_t c = 0; c < total_cells; ++c) cnt[c] = bin_start[c];
        for (size_t i = 0; i < total; ++i) {
            uint32_t c = atom_cell[i];
            uint32_t p = cnt[c];
            sorted_atoms[p] = (uint32_t)i;
            atom_sorted_idx[i] = p;
            cnt[c] = p + 1;
        }
        std::vector<V3> sorted_pos(total);
        for (size_t m = 0; m < total; ++m) sorted_pos[m] = pos[sorted_atoms[m]];

        neighbor_offsets.clear();
        neighbor_indices.clear();
        bool has_self = bin_stencil_self;
        const std::vector<int32_t>& stencil = newton ? bin_stencil_forward : bin_stencil;
        double sf_sq = skin_fraction * skin_fraction;
        for (size_t i = 0; i < nl; ++i) {
            neighbor_offsets.push_back((uint32_t)neighbor_indices.size());
            size_t my_cell = atom_cell[i];
            const V3 pi = pos[i];
            double si = cutoff_radius[i];
            auto accept = [&](size_t m, size_t j) {
                const V3& pj = sorted_pos[m];
                double dx = pj[0] - pi[0], dy = pj[1] - pi[1], dz = pj[2] - pi[2];
                double r2 = std::fma(dx, dx, std::fma(dy, dy, dz * dz));
                if (has_uniform_cutoff) return r2 < uniform_cutoff_sq;
                double sum_skin = si + cutoff_radius[j];
                return r2 < sum_skin * sum_skin * sf_sq;
            };
            if (has_self) {
                size_t cs = bin_start[my_cell], ce = bin_start[my_cell + 1];
                if (newton) {
                    for (size_t m = (size_t)atom_sorted_idx[i] + 1; m < ce; ++m)
                        if (accept(m, sorted_atoms[m])) neighbor_indices.push_back(sorted_atoms[m]);
                } else {
                    for (size_t m = cs; m < ce; ++m) {
                        uint32_t j = sorted_atoms[m];
                        if ((size_t)j == i) continue;
                        if (accept(m, j)) neighbor_indices.push_back(j);
                    }
                }
            }
            for (int32_t off : stencil) {
                if (!newton && off == 0) continue;
                size_t c = (size_t)((int32_t)my_cell + off);
                size_t s = bin_start[c], e = bin_start[c + 1];
                for (size_t m = s; m < e; ++m)
                    if (accept(m, sorted_atoms[m])) neighbor_indices.push_back(sorted_atoms[m]);
            }
        }
        neighbor_offsets.push_back((uint32_t)neighbor_indices.size());
        rebuilds += 1;
    }

    // Force phase: the tutorial's soft_repulsion_force
    // (docs/src/tutorial/write-your-own-physics.md:56-110) with K = harmonic_k.
    void phase_force() {
        if (harmonic_k == 0.0 || radius_col < 0) return;
        const Column& rc = cols[radius_col];
        size_t nl = nlocal;
        double K = harmonic_k;
        for (size_t i = 0; i < nl; ++i) {
            for (uint32_t k = neighbor_offsets[i]; k < neighbor_offsets[i + 1]; ++k) {
                size_t j = neighbor_indices[k];
                double ri = rc.data[i * rc.width], rj = rc.data[j * rc.width];
                double sum_r = ri + rj;
                double dx = pos[j][0] - pos[i][0];
                double dy = pos[j][1] - pos[i][1];
                double dz = pos[j][2] - pos[i][2];
                double dist_sq = dx * dx + dy * dy + dz * dz;
                if (dist_sq >= sum_r * sum_r || dist_sq == 0.0) continue;
                double dist = std::sqrt(dist_sq);
                double overlap = sum_r - dist;
                double inv_dist = 1.0 / dist;
                double fmag = K * overlap;
                double fx = -fmag * dx * inv_dist;
                double fy = -fmag * dy * inv_dist;
                double fz = -fmag * dz * inv_dist;
                force[i][0] += fx; force[i][1] += fy; force[i][2] += fz;
                if (newton || j < nl) {
                    force[j][0] -= fx; force[j][1] -= fy; force[j][2] -= fz;
                }
            }
        }
    }

    // Test consumer of registered columns (no reference counterpart; it plays
    // the part of a physics plugin that writes #[reverse] / #[zero] /
    // #[forward] data in its Force system, after the pair forces):
    //   every atom a (locals and ghosts): rev[a] += {0.5 x, y - z};
    //                                     zacc[a] += 0.25 x
    //   every local a:                    fwd[a][k] += 0.001 pos[a][k]
    // Each value depends on its own atom only, so any evaluation order gives
    // the same bits; the reverse fold, the zeroing and forward comm then
    // decide what the columns hold.
    int probe_rev = -1, probe_zero = -1, probe_fwd = -1;
    void column_probe() {
        size_t n = len();
        if (probe_rev >= 0) {
            Column& c = cols[probe_rev];
            for (size_t a = 0; a < n; ++a) {
                c.data[a * c.width + 0] = c.data[a * c.width + 0] + 0.5 * pos[a][0];
                c.data[a * c.width + 1] = c.data[a * c.width + 1] + (pos[a][1] - pos[a][2]);
            }
        }
        if (probe_zero >= 0) {
            Column& c = cols[probe_zero];
            for (size_t a = 0; a < n; ++a) c.data[a * c.width] = c.data[a * c.width] + 0.25 * pos[a][0];
        }
        if (probe_fwd >= 0) {
            Column& c = cols[probe_fwd];
            for (size_t a = 0; a < nlocal; ++a)
                for (int k = 0; k < 3; ++k)
                    c.data[a * c.width + k] = c.data[a * c.width + k] + 0.001 * pos[a][k];
        }
    }

    // reverse_send_force self-send path, comm.rs:867-1024 (run_if newton)
    void phase_reverse_comm() {
        if (!newton) return;
        size_t end = swaps.size();
        while (end > 0) {
            size_t start = end >= 2 ? end - 2 : 0;
            for (size_t s = start; s < end; ++s) {
                const Swap& sw = swaps[s];
                if (sw.to_proc < 0 || sw.from_proc < 0) continue;  // no neighbor (comm.rs:460)
                std::vector<double> buf;  // pack_reverse_into: force then #[reverse] columns
                for (size_t g = sw.recv_start; g < sw.recv_start + sw.recv_count; ++g) {
                    buf.push_back(force[g][0]); buf.push_back(force[g][1]); buf.push_back(force[g][2]);
                    for (auto& c : cols)
                        if (c.flags & SOIL_COL_REVERSE)
                            for (int w = 0; w < c.width; ++w) buf.push_back(c.data[g * c.width + w]);
                }
                size_t per = sw.recv_count ? buf.size() / sw.recv_count : 0;
                for (size_t k = 0; k < sw.send_indices.size(); ++k) {  // reverse_accumulate
                    size_t o = sw.send_indices[k];
                    size_t b = k * per;
                    force[o][0] += buf[b + 0]; force[o][1] += buf[b + 1]; force[o][2] += buf[b + 2];
                    size_t q = 3;
                    for (auto& c : cols)
                        if (c.flags & SOIL_COL_REVERSE)
                            for (int w = 0; w < c.width; ++w) c.data[o * c.width + w] += buf[b + q++];
                }
            }
            end = start;
        }
    }

    bool step() {
        if (!phase_deform()) return false;  // PreInitialIntegration
        phase_initial();           // InitialIntegration
        phase_decide_rebuild();    // PostInitialIntegration
        phase_remove_ghosts();
        phase_zero_forces();
        phase_shrink_wrap();       // PreExchange
        phase_pbc();
        phase_sort();              // PreNeighbor
        phase_borders();
        phase_forward_comm();
        phase_neighbor();          // Neighbor
        phase_force();             // Force
        column_probe();
        phase_reverse_comm();      // PostForce
        phase_final();             // FinalIntegration
        steps_done += 1;
        return true;
    }
};

}  // namespace

// ===========================================================================
// C API (orc_*) — the same shapes as soil_cuda.h, on host memory.
// ===========================================================================
extern "C" {

void* orc_create(const soil_box* box, const soil_neigh_cfg* cfg, double dt) {
    Sys* s = new Sys();
    for (int d = 0; d < 3; ++d) {
        s->blo[d] = box->lo[d];
        s->bhi[d] = box->hi[d];
        s->size[d] = box->hi[d] - box->lo[d];
        s->sub_lo[d] = box->lo[d];  // decompose_domain, 1x1x1 grid (domain.rs:235-296)
        s->sub_hi[d] = box->lo[d] + s->size[d] / 1.0 * 1.0;
        s->sub_len[d] = s->size[d] / 1.0;
    }
    s->dt = dt;
    s->skin_fraction = cfg->skin_fraction;
    s->bin_min_size = cfg->bin_size;
    s->every = cfg->every;
    s->check = cfg->check != 0;
    s->sort_every = cfg->sort_every;
    s->newton = cfg->newton != 0;
    s->additive_skin = cfg->additive_skin;
    return s;
}

void orc_destroy(void* h) { delete (Sys*)h; }

int orc_register_column(void* h, int32_t width, uint32_t flags) {
    Sys* s = (Sys*)h;
    if (width <= 0 || s->setup_done) return -1;
    Column c;
    c.name = "col" + std::to_string(s->cols.size());
    c.width = width;
    c.flags = flags;
    c.data.assign(s->len() * (size_t)width, 0.0);
    s->cols.push_back(c);
    return (int)s->cols.size() - 1;
}

int orc_add_atoms(void* h, uint64_t n, const uint32_t* tag, const uint32_t* type, const double* pos3,
                  const double* vel3, const double* mass, const double* cutoff,
                  const double* const* columns) {
    Sys* s = (Sys*)h;
    if (s->setup_done) return SOIL_ERR_STATE;
    size_t base = s->len();
    for (uint64_t i = 0; i < n; ++i) {
        V3 p{pos3[3 * i], pos3[3 * i + 1], pos3[3 * i + 2]};
        V3 v{vel3[3 * i], vel3[3 * i + 1], vel3[3 * i + 2]};
        s->push_atom(tag[i], type ? type[i] : 0, 0, p, v, {0, 0, 0}, cutoff[i], mass[i], 1.0 / mass[i],
                     {0, 0, 0}, false);
    }
    for (size_t c = 0; c < s->cols.size(); ++c) {
        Column& col = s->cols[c];
        col.data.resize(s->len() * (size_t)col.width, 0.0);
        if (columns && columns[c])
            for (uint64_t k = 0; k < n * (uint64_t)col.width; ++k) col.data[base * col.width + k] = columns[c][k];
    }
    s->nlocal = (uint32_t)s->len();
    return SOIL_OK;
}

int orc_setup(void* h) {
    Sys* s = (Sys*)h;
    // setup_deform panics on xy shear without periodic x and y (lib.rs:365-371)
    if (s->shear && (!s->is_periodic(0) || !s->is_periodic(1))) return SOIL_ERR_INVALID;
    s->comm_setup();
    s->neighbor_setup();
    s->setup_deform();
    s->setup_done = true;
    return SOIL_OK;
}

int orc_set_shear(void* h, double rate) {
    Sys* s = (Sys*)h;
    s->shear = true;
    s->shear_rate = rate;
    return SOIL_OK;
}

int orc_set_deform(void* h, int32_t dim, int32_t style, double a, double b, uint64_t stage) {
    Sys* s = (Sys*)h;
    if (dim < 0 || dim > 2 || style < 0 || style > 3) return SOIL_ERR_INVALID;
    s->axes[dim].style = style;
    s->axes[dim].a = a;
    s->axes[dim].b = b;
    s->axes[dim].stage = stage;
    return SOIL_OK;
}

int orc_set_boundary(void* h, const int32_t* type, double padding) {
    Sys* s = (Sys*)h;
    for (int d = 0; d < 3; ++d) {
        if (type[d] < 0 || type[d] > 2) return SOIL_ERR_INVALID;
        s->btype[d] = type[d];
    }
    s->shrink_wrap_padding = padding;
    return SOIL_OK;
}

int orc_set_deform_remap(void* h, int32_t remap) {
    ((Sys*)h)->remap = remap != 0;
    return SOIL_OK;
}

int orc_get_box(void* h, double* lo, double* hi, double* tilt) {
    Sys* s = (Sys*)h;
    for (int d = 0; d < 3; ++d) {
        lo[d] = s->blo[d];
        hi[d] = s->bhi[d];
        tilt[d] = s->tilt[d];
    }
    return SOIL_OK;
}

// Test consumer of registered columns (see column_probe); -1 disables a part.
int orc_set_column_probe(void* h, int32_t rev_col, int32_t zero_col, int32_t fwd_col) {
    Sys* s = (Sys*)h;
    const int32_t n = (int32_t)s->cols.size();
    if (rev_col >= n || zero_col >= n || fwd_col >= n) return SOIL_ERR_INVALID;
    if (rev_col >= 0 && s->cols[rev_col].width < 2) return SOIL_ERR_INVALID;
    if (fwd_col >= 0 && s->cols[fwd_col].width < 3) return SOIL_ERR_INVALID;
    s->probe_rev = rev_col;
    s->probe_zero = zero_col;
    s->probe_fwd = fwd_col;
    return SOIL_OK;
}

int orc_set_harmonic(void* h, double k, int32_t radius_col) {
    Sys* s = (Sys*)h;
    s->harmonic_k = k;
    s->radius_col = radius_col;
    return SOIL_OK;
}

int orc_step(void* h, uint64_t nsteps) {
    Sys* s = (Sys*)h;
    if (!s->setup_done) return SOIL_ERR_STATE;
    for (uint64_t k = 0; k < nsteps; ++k)
        if (!s->step()) return SOIL_ERR_INVALID;  // a deforming axis collapsed
    return SOIL_OK;
}

// per-phase entry points
int orc_phase(void* h, int which) {
    Sys* s = (Sys*)h;
    switch (which) {
        case 0:
            if (!s->phase_deform()) return SOIL_ERR_INVALID;
            break;
        case 1: s->phase_initial(); break;
        case 2: s->phase_decide_rebuild(); break;
        case 3: s->phase_remove_ghosts(); break;
        case 4: s->phase_zero_forces(); break;
        case 5: s->phase_pbc(); break;
        case 6: s->phase_sort(); break;
        case 7: s->phase_borders(); break;
        case 8: s->phase_forward_comm(); break;
        case 9: s->phase_neighbor(); break;
        case 10: s->phase_force(); s->column_probe(); break;
        case 11: s->phase_reverse_comm(); break;
        case 12: s->phase_final(); s->steps_done += 1; break;
        case 13: s->phase_shrink_wrap(); break;
        default: return SOIL_ERR_INVALID;
    }
    return SOIL_OK;
}

int orc_counts(void* h, soil_counts* o) {
    Sys* s = (Sys*)h;
    std::memset(o, 0, sizeof(*o));
    o->nlocal = s->nlocal;
    o->nghost = s->nghost;
    o->npairs = s->neighbor_indices.size();
    o->step = s->steps_done;
    o->rebuilds = s->rebuilds;
    o->sorts = s->sorts;
    o->steps_since_build = s->steps_since_build;
    o->comm_state = s->state;
    o->triclinic = s->triclinic;
    for (int d = 0; d < 3; ++d) o->bin_count[d] = s->bin_count[d];
    o->nstencil_forward = (int32_t)s->bin_stencil_forward.size();
    o->ghost_cutoff = s->ghost_cutoff;
    o->max_cutoff = s->cached_max_cutoff;
    o->tilt_xy = s->tilt[0];
    return SOIL_OK;
}

int orc_get_atoms(void* h, uint64_t first, uint64_t n, uint32_t* tag, double* pos3, double* vel3,
                  double* force3, int32_t* image3, int32_t* origin) {
    Sys* s = (Sys*)h;
    if (first + n > s->len()) return SOIL_ERR_INVALID;
    for (uint64_t k = 0; k < n; ++k) {
        size_t i = first + k;
        if (tag) tag[k] = s->tag[i];
        for (int d = 0; d < 3; ++d) {
            if (pos3) pos3[3 * k + d] = s->pos[i][d];
            if (vel3) vel3[3 * k + d] = s->vel[i][d];
            if (force3) force3[3 * k + d] = s->force[i][d];
            if (image3) image3[3 * k + d] = s->image[i][d];
        }
        if (origin) origin[k] = s->origin_index[i];
    }
    return SOIL_OK;
}

int orc_get_column(void* h, int32_t col, uint64_t first, uint64_t n, double* out) {
    Sys* s = (Sys*)h;
    if (col < 0 || (size_t)col >= s->cols.size() || first + n > s->len()) return SOIL_ERR_INVALID;
    const Column& c = s->cols[col];
    std::memcpy(out, c.data.data() + first * c.width, n * c.width * sizeof(double));
    return SOIL_OK;
}

int orc_get_neighbor(void* h, uint32_t* offsets, uint32_t* indices) {
    Sys* s = (Sys*)h;
    if (offsets) std::memcpy(offsets, s->neighbor_offsets.data(), s->neighbor_offsets.size() * 4);
    if (indices) std::memcpy(indices, s->neighbor_indices.data(), s->neighbor_indices.size() * 4);
    return SOIL_OK;
}

int orc_num_offsets(void* h) { return (int)((Sys*)h)->neighbor_offsets.size(); }

int orc_num_swaps(void* h) { return (int)((Sys*)h)->swaps.size(); }

int orc_get_swap_sends(void* h, int32_t si, uint64_t* count) {
    Sys* s = (Sys*)h;
    if (si < 0 || (size_t)si >= s->swaps.size()) return SOIL_ERR_INVALID;
    *count = s->swaps[si].send_indices.size();
    return SOIL_OK;
}

int orc_get_swap(void* h, int32_t si, uint64_t* recv_start, uint64_t* recv_count, double* off,
                 double* voff, uint32_t* send) {
    Sys* s = (Sys*)h;
    if (si < 0 || (size_t)si >= s->swaps.size()) return SOIL_ERR_INVALID;
    const Swap& w = s->swaps[si];
    if (recv_start) *recv_start = w.recv_start;
    if (recv_count) *recv_count = w.recv_count;
    for (int d = 0; d < 3; ++d) {
        if (off) off[d] = w.periodic_offset[d];
        if (voff) voff[d] = w.vel_offset[d];
    }
    if (send)
        for (size_t k = 0; k < w.send_indices.size(); ++k) send[k] = (uint32_t)w.send_indices[k];
    return SOIL_OK;
}

int orc_get_sort_perm(void* h, uint32_t* perm) {
    Sys* s = (Sys*)h;
    for (size_t k = 0; k < s->last_perm.size(); ++k) perm[k] = (uint32_t)s->last_perm[k];
    return (int)s->last_perm.size();
}

int orc_get_stencil(void* h, int32_t* fwd, int32_t* nfwd, double* origin3, double* binsize3) {
    Sys* s = (Sys*)h;
    if (nfwd) *nfwd = (int32_t)s->bin_stencil_forward.size();
    if (fwd)
        for (size_t k = 0; k < s->bin_stencil_forward.size(); ++k) fwd[k] = s->bin_stencil_forward[k];
    for (int d = 0; d < 3; ++d) {
        if (origin3) origin3[d] = s->bin_origin[d];
        if (binsize3) binsize3[d] = s->bin_size[d];
    }
    return SOIL_OK;
}

// The full stencil (used by newton-off lists) and whether the own cell is part
// of the stencil (bin_stencil_self).
int orc_get_stencil_full(void* h, int32_t* full, int32_t* nfull, int32_t* has_self) {
    Sys* s = (Sys*)h;
    if (nfull) *nfull = (int32_t)s->bin_stencil.size();
    if (full)
        for (size_t k = 0; k < s->bin_stencil.size(); ++k) full[k] = s->bin_stencil[k];
    if (has_self) *has_self = s->bin_stencil_self ? 1 : 0;
    return SOIL_OK;
}

// Direct access for known-answer tests of single functions.
int orc_set_state(void* h, int state) {
    ((Sys*)h)->state = state == 0 ? FULL_REBUILD : COMMUNICATE_ONLY;
    return SOIL_OK;
}
int orc_set_domain_tilt(void* h, double xy, double bvel_x, int triclinic) {
    Sys* s = (Sys*)h;
    s->tilt[0] = xy;
    s->bvel[0] = bvel_x;
    s->triclinic = triclinic != 0;
    return SOIL_OK;
}
int orc_set_atom_state(void* h, uint64_t i, const double* pos3, const double* vel3, const double* force3) {
    Sys* s = (Sys*)h;
    if (i >= s->len()) return SOIL_ERR_INVALID;
    for (int d = 0; d < 3; ++d) {
        if (pos3) s->pos[i][d] = pos3[d];
        if (vel3) s->vel[i][d] = vel3[d];
        if (force3) s->force[i][d] = force3[d];
    }
    return SOIL_OK;
}
int orc_x2lamda(void* h, const double* r, double* lam) {
    V3 l = ((Sys*)h)->x2lamda({r[0], r[1], r[2]});
    lam[0] = l[0]; lam[1] = l[1]; lam[2] = l[2];
    return SOIL_OK;
}
int orc_lamda2x(void* h, const double* lam, double* r) {
    V3 x = ((Sys*)h)->lamda2x({lam[0], lam[1], lam[2]});
    r[0] = x[0]; r[1] = x[1]; r[2] = x[2];
    return SOIL_OK;
}

}  // extern "C"
