// Split-precision FP64 products on the INT8 tensor cores (Ozaki scheme II: integer modular
// technique).  C = alpha * L R^T + beta * C for a left operand L (M x K) and a right operand R
// (N x K) given by element strides, so every BLAS transpose case maps onto it.
//
//   1. per row of L (column of the product) a power-of-two shift s_i puts the row into
//      integers of at most b bits: q_ik = rint(L_ik 2^s_i), |q| <= 2^b, likewise t_j for R;
//   2. q mod p_l for NMOD = 16 pairwise coprime moduli p_l <= 256 (product P ~ 2^126.4) as
//      signed bytes, written K-major;
//   3. per modulus one INT8 tensor-core GEMM (k_i8_mod_gemm, digits 1) gives
//      (q_L q_R^T) mod p_l exactly;
//   4. a symmetric-digit Garner CRT rebuilds the integer product (|.| < P/2 because
//      b = floor((log2 P - 2 - ceil(log2 K)) / 2)) and Horner-evaluates it in FP64 (exact below
//      2^53, a few ulps above), scaled back by 2^-(s_i + t_j).
// Accuracy: the quantisation error of an entry is at most 2^-b-1 of its row's largest entry,
// b = 56 at K = 2048 and 55 at K = 4096 -- finer than binary64's own rounding of that entry.
// FP64 stays for the scaling, the residues and the reconstruction; the products are INT8.
#pragma once
#include <cstdint>

#include "device.cuh"

namespace sdpxg {

constexpr int kOzMod = 16;

struct OzakiWorkspace {
  DevBuf<unsigned long long> amaxL, amaxR;  // per-line maxima of |operand| (FP64 bits)
  DevBuf<int> moduli, err;
  DevBuf<int8_t> PL, PR, PC;
  DevBuf<uint32_t> status;
  bool init = false;
};

// One split-precision product on `st` (no host synchronisation).  Element (i, k) of L at
// L[i * l_sr + k * l_sk], element (j, k) of R at R[j * r_sr + k * r_sk]; C column-major with
// leading dimension ldc.  upper_only writes only the entries i <= j.  Non-finite entries set
// SDPXG_ST_NONFINITE in ws.status.
void ozaki_gemm(OzakiWorkspace& ws, cudaStream_t st, int M, int N, int K, const double* L, long l_sr,
                long l_sk, const double* R, long r_sr, long r_sk, double alpha, double beta, double* C,
                long ldc, int upper_only);

// Integer bits b of the quantised operands for inner dimension K.
int ozaki_bits(int K);

}  // namespace sdpxg
