// FirstDim on the 5th-generation tensor cores: the database scan as an exact
// limb-split integer GEMM (tcgen05.mma kind::i8, accumulators in TMEM).
//
// For every eval slot t the scan is a matrix product over the rows i:
//   C_t[j][c] = sum_i D_t[j][i] * S_t[i][c]  (mod q2),
// j = database column, c = selection column (query b, mask or body). Residues
// are below q2 < 2^40, so each is split into five unsigned bytes and
//   D S = sum_{k,l} (d_k s_l) 2^{8(k+l)},
// 25 byte products accumulated exactly in 32-bit TMEM lanes (each sum is at
// most 5 * I * 255^2 < 2^31 for I <= 4096), then folded mod q2 once.
#pragma once
#include <cstddef>
#include <cstdint>

#include "common.cuh"

namespace via {

// Byte-plane layout of the prepared database (built once at setup):
//   [t][jt][kc][limb][128 x 64 bytes in the tensor-core K-major core-matrix order]
// jt = j / 128, kc = i / 64; every (t, jt, kc) chunk of 5 * 128 * 64 bytes is
// contiguous, so one bulk copy moves it into shared memory. Rows i >= I and
// columns j >= J are zero.
constexpr int FD_KC = 64;     // bytes of the reduction (row) dimension per chunk
constexpr int FD_MT = 128;    // database columns per MMA tile (the M dimension)
constexpr int FD_LIMBS = 5;   // bytes per residue
constexpr int FD_CHUNK = FD_LIMBS * FD_MT * FD_KC;  // 40960 bytes

struct FdPlan {
  const uint8_t* planes = nullptr;
  int I = 0, J = 0, n = 0;  // rows, columns, ring degree
  int I_pad = 0, J_pad = 0;
  DevMod m{};
  int grid = 148;  // persistent CTAs (one per SM)
  int* err = nullptr;  // device word: nonzero after a bounded wait ran out
};

inline int fd_round_up(int v, int a) { return (v + a - 1) / a * a; }
size_t fd_planes_bytes(int I, int J, int n);
bool fd_supported(int I, int n, u64 q);

// Converts rows [i0, i0 + 16) of an eval-form database held as u64 [16][J][n]
// (`stage`, rows beyond I ignored) into the byte planes.
void fd_rows_to_planes(const u64* stage, int i0, const FdPlan& p, uint8_t* planes, cudaStream_t st);

// Raises the scan kernel's shared-memory limit on the current device (once per
// device, before the first fd_scan there).
void fd_prepare_device();

// Scratch (bytes) that fd_scan needs for nq queries' split selection vectors.
size_t fd_sel_bytes(const FdPlan& p, int nq);

// out_eval[b][j] = sum_i sel_eval[b][i] (.) db[i][j] for mask and body:
// sel_eval [nq][I][2][n], out_eval [nq][J][2][n], eval form mod q2.
void fd_scan(const FdPlan& p, const u64* sel_eval, u64* out_eval, int nq, uint8_t* scratch, cudaStream_t st);

}  // namespace via
