// RA_PREC_MIXED: the Legendre transforms and the implicit solve as batched
// split-precision products on the int8 tensor cores (k_ozaki.cu).
//
// Both transforms are computed transposed, with the long, contiguous column
// index (field, r, re/im) as the product's M: the tensor-memory lanes, and so
// the epilogue threads, then walk contiguous output addresses.
// Inverse transform (StP_4d_dgp2, Legendre_Transforms.F90:968-1074), one
// product per (m, parity):  p2[theta_h][m][par][col] = sum_l P(l, theta_h) s2[row(m,l)][col]
//   A = s2^T (M = 11 fields x N_r x re/im, K = number of l of that parity):
//            digits made every step (exponent per column of s2, over l);
//   B = P    (N = N_theta/2): digits of the FP64 tables made once at set-up.
// Forward transform (PtS_4d_dgpv3, Legendre_Transforms.F90:1077-1175), per (m, parity):
//   s2[row(m,l)][col] = sum_theta iP(l, theta) p2b[m][par][theta][col]
//   A = p2b^T (M = 4 fields x N_r x re/im, K = N_theta/2): split every step;
//   B = iP^T  (N = number of l): digits of the iP rows, made once at set-up.
// Every product of a transform goes out in ONE launch (tile list ordered by K).
#include <algorithm>
#include <vector>

#include "ra_internal.h"
#include "ozaki.h"

namespace ra {

template <class T>
static void malloc_dev(T*& p, size_t count) {
    cudaError_t e = cudaMalloc(&p, count * sizeof(T));
    if (e != cudaSuccess) throw CudaError(e, "cudaMalloc", __FILE__, __LINE__);
}

template <class T>
static T* upload(Ctx& c, const std::vector<T>& v) {
    T* d = nullptr;
    malloc_dev(d, v.size());
    RA_CUDA(cudaMemcpyAsync(d, v.data(), v.size() * sizeof(T), cudaMemcpyHostToDevice, c.stream));
    return d;
}

static void plan_launch(Ctx& c, MixedPlan& p, const std::vector<OzProblem>& probs) {
    std::vector<int> tiles = ozaki_tiles(probs);
    p.d_probs = upload(c, probs);
    p.d_tiles = upload(c, tiles);
    p.ntiles = (int)(tiles.size() / 4);
}

static void free_plan(MixedPlan& p);

static void run_split_once(Ctx& c, const std::vector<OzSplitJob>& jobs, int max_rows) {
    if (jobs.empty()) return;
    OzSplitJob* d = upload(c, jobs);
    ozaki_split(c, d, (int)jobs.size(), max_rows, oz_split_kinds(jobs.data(), (int)jobs.size()));
    RA_CUDA(cudaStreamSynchronize(c.stream));
    cudaFree(d);
}

// ---------------------------------------------------------------------------
// Inverse Legendre transform
// ---------------------------------------------------------------------------
// The plan of one batched inverse transform p2 = P s2 over ncol columns (s2 rows in the
// m-major parity-sorted order, p2[theta_h][m][par][col]): the step's (s2a11 -> p2a) and the
// device-resident unit transform's.
static void build_lt_inverse(Ctx& c, MixedPlan& p, const double* s2, double* p2, int ncol) {
    const Dims& d = c.d;
    const int L = d.L, nth2 = d.nth2;
    const int nta = oz_tiles_of(ncol, OZ_HA), ntb = oz_tiles_of(nth2, OZ_HB);
    std::vector<long> aoff(2 * L + 1, 0), boff(2 * L + 1, 0);
    std::vector<int> nks(2 * L), nl(2 * L);
    for (int q = 0; q < 2 * L; ++q) {
        const int m = q >> 1, par = q & 1;
        nl[q] = par ? n_odd(m, L) : n_even(m, L);
        nks[q] = oz_ksteps(nl[q]);
        aoff[q + 1] = aoff[q] + (long)nta * nks[q] * OZ_ABLK;
        boff[q + 1] = boff[q] + (long)ntb * nks[q] * OZ_BBLK;
    }
    malloc_dev(p.d_adig, (size_t)aoff[2 * L]);
    malloc_dev(p.d_bdig, (size_t)boff[2 * L]);
    malloc_dev(p.d_ea, (size_t)2 * L * ncol);
    malloc_dev(p.d_eb, (size_t)2 * L * nth2);
    std::vector<OzSplitJob> ajobs, bjobs;
    std::vector<OzProblem> probs;
    for (int q = 0; q < 2 * L; ++q) {
        const int m = q >> 1, par = q & 1;
        const long roff = m_off(m, L) + (par ? n_even(m, L) : 0);
        double* out = p2 + (size_t)q * ncol;   // p2[theta_h][m][par][col]
        const long th_stride = 2L * L * ncol;
        if (nks[q] == 0) {   // no l of this parity: the E/O block stays zero
            RA_CUDA(cudaMemset2DAsync(out, th_stride * sizeof(double), 0, ncol * sizeof(double), nth2, c.stream));
            continue;
        }
        int8_t* adig = p.d_adig + aoff[q];
        int8_t* bdig = p.d_bdig + boff[q];
        int* ea = p.d_ea + (size_t)q * ncol;
        int* eb = p.d_eb + (size_t)q * nth2;
        // A = s2^T: rows = columns of the s2 block (contiguous), K = l; split every step
        ajobs.push_back({s2 + roff * ncol, 1L, (long)ncol, ncol, nl[q], OZ_HA, nta, nks[q], adig, ea});
        // B^T = P^T: rows theta_h (contiguous in the table), K = l; split once
        bjobs.push_back({c.d_Ptab + roff * nth2, 1L, (long)nth2, nth2, nl[q], OZ_HB, ntb, nks[q], bdig, eb});
        probs.push_back({adig, bdig, (long)nks[q] * OZ_ABLK, (long)nks[q] * OZ_BBLK, ea, eb, ncol, nth2, nks[q], out,
                         1L, th_stride});
    }
    run_split_once(c, bjobs, ntb * OZ_HB);
    p.d_jobs = upload(c, ajobs);
    p.njobs = (int)ajobs.size();
    p.max_rows = nta * OZ_HA;
    p.kinds = oz_split_kinds(ajobs.data(), p.njobs);
    plan_launch(c, p, probs);
}

static void setup_lt_inverse(Ctx& c) { build_lt_inverse(c, c.mx_inv, c.d_s2a11, c.d_p2a, c.nfa * c.d.nr * 2); }

static void run_plan(Ctx& c, MixedPlan& p) {
    ozaki_split(c, p.d_jobs, p.njobs, p.max_rows, p.kinds);
    ozaki_gemm(c, p.d_probs, p.d_tiles, p.ntiles, c.d_status);
}

void launch_lt_inverse_mixed(Ctx& c) { run_plan(c, c.mx_inv); }

// ---------------------------------------------------------------------------
// Forward Legendre transform
// ---------------------------------------------------------------------------
// The plan of one batched forward transform s2 = iP p2 over ncol columns (p2 folded,
// [m][par][theta_h][col]).
static void build_lt_forward(Ctx& c, MixedPlan& p, const double* p2, double* s2, int ncol) {
    const Dims& d = c.d;
    const int L = d.L, nth2 = d.nth2;
    const int nta = oz_tiles_of(ncol, OZ_HA), nks = oz_ksteps(nth2);
    const long ablk = (long)nta * nks * OZ_ABLK;
    std::vector<long> boff(2 * L + 1, 0);
    for (int q = 0; q < 2 * L; ++q) {
        const int m = q >> 1, par = q & 1;
        const int nl = par ? n_odd(m, L) : n_even(m, L);
        boff[q + 1] = boff[q] + (long)oz_tiles_of(nl, OZ_HB) * nks * OZ_BBLK;
    }
    malloc_dev(p.d_adig, (size_t)ablk * 2 * L);
    malloc_dev(p.d_bdig, (size_t)boff[2 * L]);
    malloc_dev(p.d_ea, (size_t)2 * L * ncol);
    malloc_dev(p.d_eb, (size_t)d.nlm);
    std::vector<OzSplitJob> ajobs, bjobs;
    std::vector<OzProblem> probs;
    int max_b = 0;
    for (int q = 0; q < 2 * L; ++q) {
        const int m = q >> 1, par = q & 1;
        const int nl = par ? n_odd(m, L) : n_even(m, L);
        if (nl == 0) continue;
        const long roff = m_off(m, L) + (par ? n_even(m, L) : 0);
        const int ntb = oz_tiles_of(nl, OZ_HB);
        max_b = std::max(max_b, ntb * OZ_HB);
        int8_t* adig = p.d_adig + (size_t)q * ablk;
        int8_t* bdig = p.d_bdig + boff[q];
        int* ea = p.d_ea + (size_t)q * ncol;
        int* eb = p.d_eb + roff;
        // A = p2b^T: rows = columns of the folded block (contiguous), K = theta_h
        ajobs.push_back({p2 + (size_t)q * nth2 * ncol, 1L, (long)ncol, ncol, nth2, OZ_HA, nta, nks, adig, ea});
        // B^T = iP rows (theta_h contiguous)
        bjobs.push_back({c.d_iPtab + roff * nth2, (long)nth2, 1L, nl, nth2, OZ_HB, ntb, nks, bdig, eb});
        probs.push_back({adig, bdig, (long)nks * OZ_ABLK, (long)nks * OZ_BBLK, ea, eb, ncol, nl, nks,
                         s2 + roff * ncol, 1L, (long)ncol});
    }
    run_split_once(c, bjobs, max_b);
    p.d_jobs = upload(c, ajobs);
    p.njobs = (int)ajobs.size();
    p.max_rows = nta * OZ_HA;
    p.kinds = oz_split_kinds(ajobs.data(), p.njobs);
    plan_launch(c, p, probs);
    RA_CUDA(cudaStreamSynchronize(c.stream));
}

static void setup_lt_forward(Ctx& c) { build_lt_forward(c, c.mx_fwd, c.d_p2b, c.d_s2b, c.nfb * c.d.nr * 2); }

void launch_lt_forward_mixed(Ctx& c) { run_plan(c, c.mx_fwd); }

// The device-resident unit transforms' split-product plans, one per direction, rebuilt when
// the operands or the column count change.
void launch_lt_unit_mixed(Ctx& c, int inverse, const double* in, double* out, int ncol) {
    UnitPlan& u = inverse ? c.unit_inv : c.unit_fwd;
    if (!u.built || u.in != in || u.out != out || u.ncol != ncol) {
        free_plan(u.plan);
        if (!c.d_status) {
            malloc_dev(c.d_status, 1);
            RA_CUDA(cudaMemsetAsync(c.d_status, 0, sizeof(int), c.stream));
        }
        if (inverse)
            build_lt_inverse(c, u.plan, in, out, ncol);
        else
            build_lt_forward(c, u.plan, in, out, ncol);
        RA_CUDA(cudaStreamSynchronize(c.stream));
        u.built = true;
        u.in = in;
        u.out = out;
        u.ncol = ncol;
    } else if (inverse) {
        // the caller may have reused the output buffer: the (m, parity) blocks without an l
        // (their zeros were written when the plan was built) are cleared again
        const int L = c.d.L, nth2 = c.d.nth2;
        for (int q = 0; q < 2 * L; ++q) {
            const int m = q >> 1;
            if (oz_ksteps((q & 1) ? n_odd(m, L) : n_even(m, L)) == 0)
                RA_CUDA(cudaMemset2DAsync(out + (size_t)q * ncol, 2L * L * ncol * sizeof(double), 0,
                                          ncol * sizeof(double), nth2, c.stream));
        }
    }
    run_plan(c, u.plan);
}

// ---------------------------------------------------------------------------
// Implicit solve (Implicit_Solve, Linear_Solve.F90:423-457): x = A_l^{-1} b per
// (system, l), the inverses' digits made at set-up and after every dt change,
// the right-hand sides' digits every step.  The K index of the linked W-P-T
// system runs over three blocks of very different size (the W, P and T
// coefficients); each block is a K segment with its own exponents, so the
// small W part keeps its relative accuracy.
// ---------------------------------------------------------------------------
static void setup_solve(Ctx& c) {
    const Dims& d = c.d;
    const int L = d.L, nr = d.nr;
    MixedPlan& p = c.mx_solve;
    const int kseg = oz_ksteps(nr);   // K-steps of one radial block
    const int nsys = c.mag ? 4 : 2;   // W-P-T, Z (and C, A with magnetism)
    long asize = 0, bsize = 0, esize_a = 0, esize_b = 0;
    for (int sys = 0; sys < nsys; ++sys) {
        const int n = sys ? nr : 3 * nr, nseg = sys ? 1 : 3;
        const int nta = oz_tiles_of(n, OZ_HA), nks = nseg * kseg;
        asize += (long)L * nta * nks * OZ_ABLK;
        esize_a += (long)L * nseg * n;
        for (int l = 0; l < L; ++l) {
            bsize += (long)oz_tiles_of(2 * (l + 1), OZ_HB) * nks * OZ_BBLK;
            esize_b += (long)nseg * 2 * (l + 1);
        }
    }
    malloc_dev(p.d_adig, (size_t)asize);
    malloc_dev(p.d_bdig, (size_t)bsize);
    malloc_dev(p.d_ea, (size_t)esize_a);
    malloc_dev(p.d_eb, (size_t)esize_b);
    std::vector<OzSplitJob> ajobs, bjobs;
    std::vector<OzProblem> probs;
    long ao = 0, bo = 0, eao = 0, ebo = 0;
    int max_a = 0, max_b = 0;
    for (int sys = 0; sys < nsys; ++sys) {
        const int n = sys ? nr : 3 * nr, nseg = sys ? 1 : 3;
        const int nta = oz_tiles_of(n, OZ_HA), nks = nseg * kseg;
        // transposed inverses: (i, k) at [k][i]
        const double* Ainv = sys == 0 ? c.d_Ainv_wpt : sys == 1 ? c.d_Ainv_z : sys == 2 ? c.d_Ainv_c : c.d_Ainv_a;
        const double* rhs = sys == 0 ? c.d_rhs_wpt : sys == 1 ? c.d_rhs_z : sys == 2 ? c.d_rhs_c : c.d_rhs_a;
        double* sol = sys == 0 ? c.d_sol_wpt : sys == 1 ? c.d_sol_z : sys == 2 ? c.d_sol_c : c.d_sol_a;
        max_a = std::max(max_a, nta * OZ_HA);
        for (int l = 0; l < L; ++l) {
            const long lstart = (long)l * (l + 1) / 2;
            const int ncol = 2 * (l + 1);
            const int ntb = oz_tiles_of(ncol, OZ_HB);
            max_b = std::max(max_b, ntb * OZ_HB);
            int8_t* adig = p.d_adig + ao;
            int8_t* bdig = p.d_bdig + bo;
            int* ea = p.d_ea + eao;   // [segment][n]
            int* eb = p.d_eb + ebo;   // [segment][ncol]
            ao += (long)nta * nks * OZ_ABLK;
            bo += (long)ntb * nks * OZ_BBLK;
            eao += (long)nseg * n;
            ebo += (long)nseg * ncol;
            for (int sg = 0; sg < nseg; ++sg) {
                // rows of A_l^{-1} restricted to the columns of block sg (K contiguous);
                // right-hand-side columns (lm, re/im) restricted to the rows of block sg
                ajobs.push_back({Ainv + (size_t)l * n * n + (size_t)sg * nr * n, 1L, (long)n, n, nr, OZ_HA, nta, kseg,
                                 adig, ea + (long)sg * n, nks, sg * kseg});
                bjobs.push_back({rhs + 2 * lstart * n + sg * nr, (long)n, 1L, ncol, nr, OZ_HB, ntb, kseg, bdig,
                                 eb + (long)sg * ncol, nks, sg * kseg});
            }
            probs.push_back({adig, bdig, (long)nks * OZ_ABLK, (long)nks * OZ_BBLK, ea, eb, n, ncol, nks,
                             sol + 2 * lstart * n, 1L, (long)n, nseg, (long)n, (long)ncol});
        }
    }
    p.d_setup_jobs = upload(c, ajobs);
    p.nsetup_jobs = (int)ajobs.size();
    p.setup_max_rows = max_a;
    p.setup_kinds = oz_split_kinds(ajobs.data(), p.nsetup_jobs);
    ozaki_split(c, p.d_setup_jobs, p.nsetup_jobs, p.setup_max_rows, p.setup_kinds);
    p.d_jobs = upload(c, bjobs);
    p.njobs = (int)bjobs.size();
    p.max_rows = max_b;
    p.kinds = oz_split_kinds(bjobs.data(), p.njobs);
    plan_launch(c, p, probs);
    RA_CUDA(cudaStreamSynchronize(c.stream));
}

void mixed_resplit_solve(Ctx& c) {
    MixedPlan& p = c.mx_solve;
    if (!p.d_setup_jobs) return;
    ozaki_split(c, p.d_setup_jobs, p.nsetup_jobs, p.setup_max_rows, p.setup_kinds);
    RA_CUDA(cudaStreamSynchronize(c.stream));
}

void launch_solve_mixed(Ctx& c) {
    MixedPlan& p = c.mx_solve;
    ozaki_split(c, p.d_jobs, p.njobs, p.max_rows, p.kinds);
    ozaki_gemm(c, p.d_probs, p.d_tiles, p.ntiles, c.d_status);
}

void mixed_setup(Ctx& c) {
    if (!c.d_status) {
        malloc_dev(c.d_status, 1);
        RA_CUDA(cudaMemsetAsync(c.d_status, 0, sizeof(int), c.stream));
    }
    setup_lt_inverse(c);
    setup_lt_forward(c);
    if (c.mixed_solve) setup_solve(c);
}

static void free_plan(MixedPlan& p) {
    if (p.d_adig) cudaFree(p.d_adig);
    if (p.d_bdig) cudaFree(p.d_bdig);
    if (p.d_ea) cudaFree(p.d_ea);
    if (p.d_eb) cudaFree(p.d_eb);
    if (p.d_probs) cudaFree(p.d_probs);
    if (p.d_tiles) cudaFree(p.d_tiles);
    if (p.d_jobs) cudaFree(p.d_jobs);
    if (p.d_setup_jobs) cudaFree(p.d_setup_jobs);
    p = MixedPlan{};
}

void mixed_release(Ctx& c) {
    free_plan(c.mx_inv);
    free_plan(c.mx_fwd);
    free_plan(c.unit_inv.plan);
    free_plan(c.unit_fwd.plan);
    free_plan(c.mx_solve);
}

}  // namespace ra
