// Checkpoint files in the reference's format (Write_Checkpoint / Read_Checkpoint,
// src/Physics/Checkpointing.F90:143-801, checkpoint_version = 2), host code only.
//
// A checkpoint is a directory holding
//   W P T Z (C A)            the equation-set RHS (the solution's Chebyshev coefficients)
//   WAB PAB TAB ZAB (CAB AAB) the Adams-Bashforth terms (on the radial grid)
//   boundary_conditions      bc_values: radial slot 2(i-1)+1 / 2(i-1)+2 = top / bottom of field i
//   grid_etc                 Fortran stream: int32 314 (endian tag), int32 version (2),
//                            int32 n_r, int32 grid_type (2: Chebyshev), int32 l_max,
//                            float64 dt, float64 new_dt, float64 radius[n_r],
//                            float64 elapsed_time, int32 iteration
// Every field file is n_r (l_max+1)(l_max+2) float64 (the size Read_Checkpoint
// checks, :410-420): the real parts, then the imaginary parts; within each, one
// chunk per radial index, each chunk the (l, m) pairs m-major with l fastest
// (m = 0: l = 0..l_max; m = 1: l = 1..l_max; ...), as Spectral_Prep caches them
// (src/IO/Parallel_IO.F90:973-1047) and the reference's own reader takes them
// apart (post_processing/rayleigh_diagnostics.py checkpoint_read).
#include <cerrno>
#include <cmath>
#include <cstdint>
#include <cstdio>
#include <cstring>
#include <string>
#include <sys/stat.h>
#include <vector>

#include "ra_internal.h"

namespace {

// our layout: Fortran (n_r, 2, n_lm), lm = l (l + 1) / 2 + m  <->  the file's [2][n_r][m-major triangle]
void to_file_order(const double* field, int n_r, int l_max, std::vector<double>& out) {
    const int L = l_max + 1;
    const long ntri = (long)L * (L + 1) / 2;
    out.assign((size_t)2 * n_r * ntri, 0.0);
    for (int ri = 0; ri < 2; ++ri)
        for (int r = 0; r < n_r; ++r) {
            double* chunk = out.data() + ((size_t)ri * n_r + r) * ntri;
            long k = 0;
            for (int m = 0; m < L; ++m)
                for (int l = m; l < L; ++l)
                    chunk[k++] = field[((size_t)ra::lm_index(l, m) * 2 + ri) * n_r + r];
        }
}

void from_file_order(const std::vector<double>& in, int n_r, int l_max, double* field) {
    const int L = l_max + 1;
    const long ntri = (long)L * (L + 1) / 2;
    for (int ri = 0; ri < 2; ++ri)
        for (int r = 0; r < n_r; ++r) {
            const double* chunk = in.data() + ((size_t)ri * n_r + r) * ntri;
            long k = 0;
            for (int m = 0; m < L; ++m)
                for (int l = m; l < L; ++l)
                    field[((size_t)ra::lm_index(l, m) * 2 + ri) * n_r + r] = chunk[k++];
        }
}

bool write_bytes(const std::string& path, const void* data, size_t bytes) {
    FILE* f = std::fopen(path.c_str(), "wb");
    if (!f) return false;
    const bool ok = std::fwrite(data, 1, bytes, f) == bytes;
    return std::fclose(f) == 0 && ok;
}

bool read_bytes(const std::string& path, std::vector<unsigned char>& out) {
    FILE* f = std::fopen(path.c_str(), "rb");
    if (!f) return false;
    out.clear();
    unsigned char buf[1 << 16];
    size_t n;
    while ((n = std::fread(buf, 1, sizeof(buf), f)) > 0) out.insert(out.end(), buf, buf + n);
    std::fclose(f);
    return true;
}

const char* kNames[6] = {"W", "P", "T", "Z", "C", "A"};

int last_err(ra_ctx* ctx, const std::string& msg, int code) {
    if (ctx) ctx->c.err = msg;
    return code;
}

}  // namespace

extern "C" {

int ra_checkpoint_write_field(const char* path, int n_r, int l_max, const double* field) {
    if (!path || !field || n_r < 1 || l_max < 0) return RA_ERR_ARG;
    std::vector<double> buf;
    to_file_order(field, n_r, l_max, buf);
    return write_bytes(path, buf.data(), buf.size() * sizeof(double)) ? RA_OK : RA_ERR_ARG;
}

int ra_checkpoint_read_field(const char* path, int n_r, int l_max, double* field) {
    if (!path || !field || n_r < 1 || l_max < 0) return RA_ERR_ARG;
    std::vector<unsigned char> raw;
    if (!read_bytes(path, raw)) return RA_ERR_ARG;
    const size_t want = (size_t)n_r * (l_max + 1) * (l_max + 2) * sizeof(double);
    if (raw.size() != want) return RA_ERR_ARG;   // wrong size: corrupted or another grid (Checkpointing.F90:410-420)
    std::vector<double> buf(raw.size() / sizeof(double));
    std::memcpy(buf.data(), raw.data(), raw.size());
    from_file_order(buf, n_r, l_max, field);
    return RA_OK;
}

int ra_write_checkpoint(ra_ctx* ctx, const char* dir, double elapsed_time) {
    if (!ctx || ctx->c.d.L == 0 || !ctx->c.have_state) return RA_ERR_STATE;
    if (!dir) return RA_ERR_ARG;
    ra::Ctx& c = ctx->c;
    const int nr = c.d.nr, lmax = c.d.lmax;
    const size_t nlm = (size_t)c.d.nlm, plane = nlm * 2 * nr;
    if (::mkdir(dir, 0755) != 0 && errno != EEXIST)
        return last_err(ctx, std::string("cannot create checkpoint directory ") + dir, RA_ERR_ARG);
    // the state through the public exchange (one synchronised copy each)
    std::vector<double> wpt(3 * plane), z(plane), ab(4 * plane), cm, am, abm;
    int rc = ra_get_state(ctx, wpt.data(), z.data(), ab.data());
    if (rc != RA_OK) return rc;
    const int nf = c.mag ? 6 : 4;
    if (c.mag) {
        cm.resize(plane);
        am.resize(plane);
        abm.resize(2 * plane);
        rc = ra_get_magnetic_state(ctx, cm.data(), am.data(), abm.data());
        if (rc != RA_OK) return rc;
    }
    // wpt is (3 n_r, 2, n_lm): split into W, P, T fields of (n_r, 2, n_lm)
    std::vector<std::vector<double>> fields(nf, std::vector<double>(plane));
    for (size_t lm = 0; lm < nlm; ++lm)
        for (int ri = 0; ri < 2; ++ri)
            for (int b = 0; b < 3; ++b)
                std::memcpy(&fields[b][(lm * 2 + ri) * nr], &wpt[((lm * 2 + ri) * 3 + b) * nr], nr * sizeof(double));
    fields[3] = z;
    if (c.mag) {
        fields[4] = cm;
        fields[5] = am;
    }
    const std::string d(dir);
    for (int i = 0; i < nf; ++i) {
        if (ra_checkpoint_write_field((d + "/" + kNames[i]).c_str(), nr, lmax, fields[i].data()) != RA_OK)
            return last_err(ctx, "cannot write checkpoint field " + std::string(kNames[i]), RA_ERR_ARG);
        const double* abi = i < 4 ? &ab[(size_t)i * plane] : &abm[(size_t)(i - 4) * plane];
        if (ra_checkpoint_write_field((d + "/" + kNames[i] + "AB").c_str(), nr, lmax, abi) != RA_OK)
            return last_err(ctx, "cannot write checkpoint field " + std::string(kNames[i]) + "AB", RA_ERR_ARG);
    }
    // boundary values: the caller's (ra_set_bc_mask) or the built-in ones (only l = 0 T)
    std::vector<double> bcv((size_t)4 * nlm * 4, 0.0);   // [eq][lm][re/im][top/bottom]
    if (c.d_bcval) {
        if (cudaMemcpy(bcv.data(), c.d_bcval, bcv.size() * sizeof(double), cudaMemcpyDeviceToHost) != cudaSuccess)
            return last_err(ctx, "cannot read the boundary values", RA_ERR_CUDA);
    } else {
        const double s4pi = std::sqrt(4.0 * M_PI);
        bcv[((size_t)2 * nlm + 0) * 4 + 0] = (c.cfg.fix_tvar_top ? c.cfg.t_top : c.cfg.dtdr_top) * s4pi;
        bcv[((size_t)2 * nlm + 0) * 4 + 1] = (c.cfg.fix_tvar_bottom ? c.cfg.t_bottom : c.cfg.dtdr_bottom) * s4pi;
    }
    std::vector<double> bfield(plane, 0.0);   // radial slot 2i: top, 2i + 1: bottom of field i
    for (int e = 0; e < 4; ++e)
        for (size_t lm = 0; lm < nlm; ++lm)
            for (int ri = 0; ri < 2; ++ri)
                for (int tb = 0; tb < 2; ++tb)
                    bfield[(lm * 2 + ri) * nr + 2 * e + tb] = bcv[(((size_t)e * nlm + lm) * 2 + ri) * 2 + tb];
    if (ra_checkpoint_write_field((d + "/boundary_conditions").c_str(), nr, lmax, bfield.data()) != RA_OK)
        return last_err(ctx, "cannot write checkpoint boundary conditions", RA_ERR_ARG);
    // grid_etc
    std::vector<unsigned char> g;
    auto put = [&](const void* p, size_t n) {
        const unsigned char* b = static_cast<const unsigned char*>(p);
        g.insert(g.end(), b, b + n);
    };
    // grid_type 2: Chebyshev, 1: finite differences (ProblemSize.F90:60, 537)
    const int32_t tag = 314, version = 2, n_r32 = nr, grid_type = c.cfg.chebyshev ? 2 : 1, l_max32 = lmax;
    const int32_t iter = c.iteration - 1;   // the last completed step
    const double dt = c.old_dt, new_dt = c.dt;
    put(&tag, 4);
    put(&version, 4);
    put(&n_r32, 4);
    put(&grid_type, 4);
    put(&l_max32, 4);
    put(&dt, 8);
    put(&new_dt, 8);
    put(c.rad.radius.data(), (size_t)nr * 8);
    put(&elapsed_time, 8);
    put(&iter, 4);
    if (!write_bytes(d + "/grid_etc", g.data(), g.size()))
        return last_err(ctx, "cannot write checkpoint grid_etc", RA_ERR_ARG);
    return RA_OK;
}

int ra_read_checkpoint(ra_ctx* ctx, const char* dir, int* iteration, double* elapsed_time) {
    if (!ctx || ctx->c.d.L == 0) return RA_ERR_STATE;
    if (!dir) return RA_ERR_ARG;
    ra::Ctx& c = ctx->c;
    const int nr = c.d.nr, lmax = c.d.lmax;
    const size_t nlm = (size_t)c.d.nlm, plane = nlm * 2 * nr;
    const std::string d(dir);
    std::vector<unsigned char> g;
    if (!read_bytes(d + "/grid_etc", g)) return last_err(ctx, "cannot open " + d + "/grid_etc", RA_ERR_ARG);
    size_t off = 0;
    auto get = [&](void* p, size_t n) {
        if (off + n > g.size()) return false;
        std::memcpy(p, g.data() + off, n);
        off += n;
        return true;
    };
    int32_t tag = 0, version = 0, n_r_old = 0, grid_type = 0, l_max_old = 0, iter = 0;
    double dt = 0, new_dt = 0, t = 0;
    if (!get(&tag, 4) || tag != 314) return last_err(ctx, "grid_etc: endian check failed", RA_ERR_ARG);
    bool ok = get(&version, 4) && get(&n_r_old, 4) && get(&grid_type, 4) && get(&l_max_old, 4) && get(&dt, 8) &&
              get(&new_dt, 8);
    if (!ok || version != 2) return last_err(ctx, "grid_etc: not a version-2 checkpoint", RA_ERR_ARG);
    if (n_r_old != nr || l_max_old != lmax || grid_type != (c.cfg.chebyshev ? 2 : 1))
        return last_err(ctx, "checkpoint grid (n_r " + std::to_string(n_r_old) + ", l_max " +
                                 std::to_string(l_max_old) + ", grid_type " + std::to_string(grid_type) +
                                 ") differs from the context's; interpolation is not provided", RA_ERR_ARG);
    std::vector<double> rad(nr);
    ok = get(rad.data(), (size_t)nr * 8) && get(&t, 8) && get(&iter, 4);
    if (!ok) return last_err(ctx, "grid_etc is truncated", RA_ERR_ARG);
    const int nf = c.mag ? 6 : 4;
    std::vector<std::vector<double>> fields(2 * nf, std::vector<double>(plane));
    for (int i = 0; i < 2 * nf; ++i) {
        const std::string name = std::string(kNames[i % nf]) + (i < nf ? "" : "AB");
        if (ra_checkpoint_read_field((d + "/" + name).c_str(), nr, lmax, fields[i].data()) != RA_OK)
            return last_err(ctx, "checkpoint field " + name + " is missing or has the wrong size", RA_ERR_ARG);
    }
    std::vector<double> wpt(3 * plane), ab(4 * plane);
    for (size_t lm = 0; lm < nlm; ++lm)
        for (int ri = 0; ri < 2; ++ri)
            for (int b = 0; b < 3; ++b)
                std::memcpy(&wpt[((lm * 2 + ri) * 3 + b) * nr], &fields[b][(lm * 2 + ri) * nr], nr * sizeof(double));
    for (int i = 0; i < 4; ++i) std::memcpy(&ab[(size_t)i * plane], fields[nf + i].data(), plane * sizeof(double));
    // the step sizes: dt was the last step's, new_dt the next one's (Reset_Linear_Equations if it differs)
    if (!(dt > 0) || !(new_dt > 0)) return last_err(ctx, "grid_etc: non-positive time step", RA_ERR_ARG);
    if (new_dt != c.dt) {
        const int rc = ra_set_dt(ctx, new_dt);
        if (rc != RA_OK) return rc;
    }
    int rc = ra_put_state(ctx, wpt.data(), fields[3].data(), ab.data(), iter + 1);
    if (rc != RA_OK) return rc;
    if (c.mag) {
        std::vector<double> abm(2 * plane);
        std::memcpy(abm.data(), fields[nf + 4].data(), plane * sizeof(double));
        std::memcpy(abm.data() + plane, fields[nf + 5].data(), plane * sizeof(double));
        rc = ra_put_magnetic_state(ctx, fields[4].data(), fields[5].data(), abm.data());
        if (rc != RA_OK) return rc;
    }
    c.old_dt = dt;   // the AB2 factors of the next step use the checkpoint's last step
    // boundary values, when the file is there (the built-in ones otherwise)
    std::vector<double> bfield(plane);
    if (ra_checkpoint_read_field((d + "/boundary_conditions").c_str(), nr, lmax, bfield.data()) == RA_OK) {
        std::vector<double> bcv((size_t)4 * nlm * 4);
        for (int e = 0; e < 4; ++e)
            for (size_t lm = 0; lm < nlm; ++lm)
                for (int ri = 0; ri < 2; ++ri)
                    for (int tb = 0; tb < 2; ++tb)
                        bcv[(((size_t)e * nlm + lm) * 2 + ri) * 2 + tb] = bfield[(lm * 2 + ri) * nr + 2 * e + tb];
        rc = ra_set_bc_mask(ctx, bcv.data());
        if (rc != RA_OK) return rc;
    }
    if (iteration) *iteration = iter;
    if (elapsed_time) *elapsed_time = t;
    return RA_OK;
}

}  // extern "C"
