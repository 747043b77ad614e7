// Split-precision (Ozaki) tensor-core products: shared declarations.
#pragma once

#include <cstdint>
#include <vector>

namespace ra {

struct Ctx;

constexpr int OZ_S = 5;   // balanced base-256 int8 digits per operand (15 digit products)
// int32 accumulators stay exact while K * 128^2 * OZ_S < 2^31
constexpr int OZ_MAX_K = 20000;
constexpr int OZ_HA = 128;   // rows of an A tile (output rows, TMEM lanes)
constexpr int OZ_HB = 96;    // rows of a B^T tile (output columns)
constexpr int OZ_BK = 32;    // K per MMA step (int8)
constexpr int OZ_ABLK = OZ_S * OZ_HA * OZ_BK;   // bytes of one K-step of an A row tile, all digits
constexpr int OZ_BBLK = OZ_S * OZ_HB * OZ_BK;   // same for B

// Digit operands are stored TILED: row tile rt (H rows) and K-step ks form one
// contiguous block of OZ_S*H*32 bytes at (rt*nks + ks) * OZ_S*H*32, laid out
// [digit s][16-byte K chunk kc][row][16 bytes] -- the tensor cores' K-major
// no-swizzle "core matrix" layout, so one bulk copy stages a whole K-step.
//
// One product C = A B of a batch: A as digit row tiles (rows = output rows,
// exponents ea[M]), B as digit row tiles of B^T (rows = output columns,
// exponents eb[N]); C(i, j) is written to C[i*c_m + j*c_n] in FP64.
// K may be cut into nseg equal segments of nks/nseg K-steps, each with its
// own exponents (ea + s*ea_seg, eb + s*eb_seg): their products are
// accumulated separately and summed in FP64, so that operands whose K range
// joins blocks of very different size keep each block's relative accuracy.
// nseg = 0 means one segment.
struct OzProblem {
    const int8_t* A;
    const int8_t* B;
    long a_tile, b_tile;   // bytes between consecutive row tiles (nks * block)
    const int* ea;
    const int* eb;
    int M, N, nks;
    double* C;
    long c_m, c_n;
    int nseg;
    long ea_seg, eb_seg;
};

// One split job: rows i < R of X (element (i, k) at X[i*sr + k*sk], k < K)
// become tiled digit rows with tile height H (nrt row tiles, nks K-steps;
// zero digits past R and K) and exponents e[i] (0 for an all-zero row).
// The job's K-steps land at K-step ks0 + ks of row tiles that hold kstride
// K-steps each (kstride = 0: the job's own nks), so that the segments of one
// operand can be split separately.
struct OzSplitJob {
    const double* X;
    long sr, sk;
    int R, K, H, nrt, nks;
    int8_t* out;
    int* e;
    int kstride, ks0;
};

// Jobs with contiguous K runs (sk == 1) and jobs with contiguous rows go to two
// kernels; kinds says which of the two a job list holds.
constexpr int OZ_SPLIT_KMAJOR = 1, OZ_SPLIT_ROWS = 2;
int oz_split_kinds(const OzSplitJob* jobs, int njobs);
void ozaki_split(Ctx& c, const OzSplitJob* d_jobs, int njobs, int max_rows,
                 int kinds = OZ_SPLIT_KMAJOR | OZ_SPLIT_ROWS);
void ozaki_gemm(Ctx& c, const OzProblem* d_probs, const int* d_tiles, int ntiles, int* d_status);
std::vector<int> ozaki_tiles(const std::vector<OzProblem>& probs);
inline int oz_tiles_of(int rows, int h) { return (rows + h - 1) / h; }
inline int oz_ksteps(int k) { return (k + OZ_BK - 1) / OZ_BK; }

}  // namespace ra
