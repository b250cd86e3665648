// restart.cu — checkpoints in the reference's restart wire format.
//
// write_restart (soil_print/src/lib.rs:1390-1445) serialises a RestartData
// (soil_print/src/lib.rs:318-418) with bincode 1's default encoding: fields in
// declaration order, little-endian, fixed-width integers, usize as u64, every
// Vec prefixed by its u64 length, fixed arrays without a prefix.  Only the
// locals are written, in their current order.  The registered columns travel
// in atom_data_buffers, one buffer per column in registration order, each
// atom's values in a row (registry pack order, atom.rs:353-365).  The legacy
// rotational fields are written empty, as the reference does.
//
// read_restart (soil_print/src/lib.rs:1527-1625) repopulates the atoms: tag,
// type, positions, velocities, forces, mass (inv_mass = 1/mass), cutoff
// radius and the columns; image flags and ghosts start empty.
#include <cstring>
#include <vector>

#include "sys_internal.cuh"

using namespace soil_host;

namespace {

struct Writer {
    uint8_t* p;
    uint64_t cap;
    uint64_t len = 0;
    void raw(const void* d, uint64_t n) {
        if (p && len + n <= cap) std::memcpy(p + len, d, n);
        len += n;
    }
    void u64(uint64_t v) { raw(&v, 8); }
    void f64(double v) { raw(&v, 8); }
    template <class T>
    void vec(const std::vector<T>& v) {
        u64(v.size());
        raw(v.data(), v.size() * sizeof(T));
    }
};

struct Reader {
    const uint8_t* p;
    uint64_t len;
    uint64_t at = 0;
    bool ok = true;
    bool raw(void* d, uint64_t n) {
        if (!ok || n > len - at) return ok = false;
        if (d) std::memcpy(d, p + at, n);
        at += n;
        return true;
    }
    uint64_t u64() {
        uint64_t v = 0;
        raw(&v, 8);
        return v;
    }
    double f64() {
        double v = 0.0;
        raw(&v, 8);
        return v;
    }
    template <class T>
    std::vector<T> vec(uint64_t elem_bytes = sizeof(T)) {
        const uint64_t n = u64();
        std::vector<T> v;
        if (!ok || n > (len - at) / elem_bytes) {
            ok = false;
            return v;
        }
        v.resize(n * (elem_bytes / sizeof(T)));
        raw(v.data(), n * elem_bytes);
        return v;
    }
};

int fetch(soil_sys* s, const void* dev, void* host, uint64_t bytes) {
    if (!bytes) return SOIL_OK;
    CK(cudaMemcpyAsync(host, dev, bytes, cudaMemcpyDeviceToHost, s->st));
    return SOIL_OK;
}

}  // namespace

extern "C" {

int soil_sys_save_restart(soil_sys* s, uint64_t total_cycle, uint8_t* buf, uint64_t cap,
                          uint64_t* len) {
    if (!s || !len) return SOIL_ERR_INVALID;
    if (s->pending_final) {  // the reference writes after FinalIntegration
        launch_final(s->st, s->nlocal, s->A, s->dt);
        s->pending_final = false;
        TRY(check_launch(s));
    }
    const uint64_t n = s->nlocal;
    std::vector<uint32_t> tag(n), type(n);
    std::vector<double> col[11];
    double* const planes[11] = {s->A.x,  s->A.y,  s->A.z,    s->A.vx,  s->A.vy, s->A.vz,
                                s->A.fx, s->A.fy, s->A.fz, s->A.mass, s->A.cut};
    for (int k = 0; k < 11; ++k) {
        col[k].resize(n);
        TRY(fetch(s, planes[k], col[k].data(), n * 8));
    }
    TRY(fetch(s, s->A.tag, tag.data(), n * 4));
    TRY(fetch(s, s->A.type, type.data(), n * 4));
    std::vector<std::vector<double>> planes_host;
    for (const ColMeta& m : s->cols)
        for (int w = 0; w < m.width; ++w) {
            planes_host.emplace_back(n);
            TRY(fetch(s, s->A.planes[m.plane0 + w], planes_host.back().data(), n * 8));
        }
    TRY(sync(s));
    Writer wr{buf, cap};
    wr.u64(n);            // natoms (one rank: every atom is local)
    wr.u64(total_cycle);  // usize
    wr.f64(s->dt);
    wr.vec(tag);
    wr.vec(type);
    for (int k = 0; k < 11; ++k) wr.vec(col[k]);  // pos_xyz, vel_xyz, force_xyz, mass, cutoff
    wr.u64(s->cols.size());                     // atom_data_buffers
    size_t q = 0;
    for (const ColMeta& m : s->cols) {
        wr.u64(n * (uint64_t)m.width);
        for (uint64_t i = 0; i < n; ++i)
            for (int w = 0; w < m.width; ++w) wr.f64(planes_host[q + w][i]);
        q += m.width;
    }
    for (int k = 0; k < 9; ++k) wr.u64(0);  // omega_xyz, torque_xyz, ang_mom_xyz
    wr.u64(0);                              // quaternion
    *len = wr.len;
    if (buf && wr.len > cap)
        return fail(s->ctx, SOIL_ERR_CAPACITY, "restart needs %llu bytes, buffer holds %llu",
                    (unsigned long long)wr.len, (unsigned long long)cap);
    return SOIL_OK;
}

int soil_sys_load_restart(soil_sys* s, const uint8_t* buf, uint64_t len, uint64_t* total_cycle) {
    if (!s || !buf) return SOIL_ERR_INVALID;
    if (s->setup_done || s->nlocal)
        return fail(s->ctx, SOIL_ERR_STATE, "load a restart into a system with no atoms, before setup");
    Reader rd{buf, len};
    const uint64_t natoms = rd.u64();
    const uint64_t cycle = rd.u64();
    const double dt = rd.f64();
    std::vector<uint32_t> tag = rd.vec<uint32_t>(), type = rd.vec<uint32_t>();
    std::vector<double> col[11];
    for (int k = 0; k < 11; ++k) col[k] = rd.vec<double>();
    const uint64_t nbuf = rd.u64();
    std::vector<std::vector<double>> bufs;
    for (uint64_t b = 0; rd.ok && b < nbuf && b <= s->cols.size(); ++b) bufs.push_back(rd.vec<double>());
    for (int k = 0; k < 9; ++k) rd.vec<double>();  // legacy rotational fields: read, unused
    rd.vec<double>(32);                            // quaternion: [f64; 4] each
    if (!rd.ok) return fail(s->ctx, SOIL_ERR_INVALID, "restart data is truncated or malformed");
    const uint64_t n = tag.size();
    bool same = type.size() == n && natoms == n;
    for (int k = 0; k < 11; ++k) same = same && col[k].size() == n;
    if (!same) return fail(s->ctx, SOIL_ERR_INVALID, "restart vectors disagree on the atom count");
    if (bufs.size() != s->cols.size())
        return fail(s->ctx, SOIL_ERR_INVALID, "restart holds %llu column buffers, %zu registered",
                    (unsigned long long)bufs.size(), s->cols.size());
    for (size_t c = 0; c < s->cols.size(); ++c)
        if (bufs[c].size() != n * (uint64_t)s->cols[c].width)
            return fail(s->ctx, SOIL_ERR_INVALID, "restart column %zu has %zu values, expected %llu", c,
                        bufs[c].size(), (unsigned long long)(n * s->cols[c].width));
    std::vector<double> pos(3 * n), vel(3 * n);
    for (uint64_t i = 0; i < n; ++i)
        for (int d = 0; d < 3; ++d) {
            pos[3 * i + d] = col[d][i];
            vel[3 * i + d] = col[3 + d][i];
        }
    std::vector<const double*> cp(s->cols.size());
    for (size_t c = 0; c < cp.size(); ++c) cp[c] = bufs[c].data();
    TRY(soil_sys_add_atoms(s, n, tag.data(), type.data(), pos.data(), vel.data(), col[9].data(),
                           col[10].data(), cp.empty() ? nullptr : cp.data()));
    CK(cudaMemcpyAsync(s->A.fx, col[6].data(), n * 8, cudaMemcpyHostToDevice, s->st));
    CK(cudaMemcpyAsync(s->A.fy, col[7].data(), n * 8, cudaMemcpyHostToDevice, s->st));
    CK(cudaMemcpyAsync(s->A.fz, col[8].data(), n * 8, cudaMemcpyHostToDevice, s->st));
    TRY(sync(s));
    s->dt = dt;
    s->steps_done = cycle;
    if (total_cycle) *total_cycle = cycle;
    return SOIL_OK;
}

}  // extern "C"
