// Split-precision (Ozaki) tensor-core products: shared declarations.
#pragma once

#include <cstdint>
#include <vector>

namespace ra {

struct Ctx;

constexpr int OZ_S = 6;   // int8 digits per operand (21 digit products)
// int32 accumulators stay exact while K * 127^2 * OZ_S < 2^31
constexpr int OZ_MAX_K = 20000;

// One product C = A B of a batch.  A is given as OZ_S int8 digit slices
// A + s*a_slice, each [rows padded to 128][kpad] (K-major), with row exponents
// ea[M]; B likewise as slices of B^T, [cols padded to 64][kpad], exponents eb[N].
// C(i, j) is written to C[i*c_m + j*c_n] in FP64.
struct OzProblem {
    const int8_t* A;
    const int8_t* B;
    long a_slice, b_slice;
    const int* ea;
    const int* eb;
    int M, N, kpad;
    double* C;
    long c_m, c_n;
};

void ozaki_split(Ctx& c, const double* X, long si, long sk, int R, int K, int rpad, int kpad, int8_t* out, long slice,
                 int* e);
void ozaki_gemm(Ctx& c, const OzProblem* d_probs, const int* d_tiles, int ntiles, int* d_status);
std::vector<int> ozaki_tiles(const std::vector<OzProblem>& probs);
int oz_round_m(int m);
int oz_round_n(int n);
int oz_round_k(int k);

}  // namespace ra
