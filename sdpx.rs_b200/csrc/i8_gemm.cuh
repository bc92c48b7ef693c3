// Modular INT8 tensor-core GEMM (tcgen05.mma kind::i8) shared by the exact RNS products of
// MpFloat matrices and the split-precision (Ozaki-II) FP64 products.
//
// For every modulus p_l (l < L) it forms the integer product of two residue matrices and reduces
// it modulo p_l in the epilogue:
//
//   digits 1: residues are single signed bytes, A_l (M x K) and B_l (N x K);
//             out_l = (A_l B_l^T) mod p_l as a signed byte in [-(p_l-1)/2, p_l/2]
//   digits 2: residues r = lo + 256 hi with signed-byte digits, A_l = (A_l0, A_l1), B_l likewise;
//             out_l = (D0 + 2^8 D1 + 2^16 D2) mod p_l in [0, p_l) as int32, with
//             D0 = A_l0 B_l0^T, D1 = A_l0 B_l1^T + A_l1 B_l0^T, D2 = A_l1 B_l1^T
//             (accumulate != 0 adds the previous residue: K split into chunks)
//
// Exactness: every D accumulates products of bytes in INT32 (|byte x byte| <= 2^14), exact for
// K <= 2^17 per call.  Operand layout: int8 planes, K contiguous ("K-major"), plane (l, d) of A
// at rows [(l*digits + d) * Mpad, ...+Mpad) of one (L*digits*Mpad) x Kld byte matrix, B alike
// with Npad; Mpad a multiple of 128, Npad of the tile width (256 for digits 1, 128 for 2), Kld
// of 128, padding zero.  Output planes: column-major m x n per modulus (entry (i, j) at
// l * plane + j * m + i), only i < m, j < n written.
#pragma once
#include <cstdint>
#include <string>

#include <cuda_runtime.h>

namespace sdpxg {

struct I8GemmArgs {
  int Mpad = 0, Npad = 0;            // padded operand row extents (see above)
  int Kld = 0;                       // bytes per operand row (the planes' padded K, a multiple of 128)
  int k0 = 0, Kpad = 0;              // this call's K range [k0, k0 + Kpad), multiples of 128
  int m = 0, n = 0;                  // output extent written
  int L = 0;                         // moduli
  const int* moduli = nullptr;       // device, L entries, 2 <= p < 2^15 (digits 2) or <= 256
  int upper_only = 0;                // skip tiles strictly below the diagonal (i > j everywhere)
  int accumulate = 0;                // digits 2: out = (out + new) mod p
  void* out = nullptr;               // int32 (digits 2) or int8 (digits 1) residue planes
  long plane = 0;                    // elements per output plane (>= m * n)
  int* err = nullptr;                // device word: bit 0 set when a bounded wait gave up
};

// Tile width (N per CTA) for each digit count.
constexpr int i8_tile_n(int digits) { return digits == 1 ? 256 : 128; }

// Launch the modular GEMM on `st`.  A and B are the device byte planes described above.  Throws
// (CudaError / invalid_argument) on a bad shape or a tensor-map failure.
void launch_i8_gemm(int digits, const int8_t* A, const int8_t* B, const I8GemmArgs& args,
                    cudaStream_t st);

// Measurement hooks: on != 0 times every later launch with CUDA events (synchronising) and
// resets the totals; i8_times reads milliseconds, INT8 operations executed (padded tiles),
// algorithmic INT8 operations (2 m n K per digit pair and modulus) and the launch count.
void i8_timing(int on);
void i8_times(double* ms, double* ops, double* alg_ops, uint64_t* count);
// Tile configuration of later launches: -1 autotuned (default), 0, 1 or 2 a fixed variant; and
// the autotuner's table (one line per shape class: the chosen variant and every timing).
void i8_set_config(int variant);
std::string i8_tuning_table();

}  // namespace sdpxg
