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
#include <utility>
#include <vector>

#include "common.cuh"

namespace via {

// Byte-plane layout of the prepared database (built once at setup):
//   [t][jt][kc][limb][128 x 64 bytes in the tensor-core K-major core-matrix order]
// jt = j / 128, kc = i / 64; every (t, jt, kc) chunk (5 * 128 * 64 bytes, or
// the packed layout below) is contiguous, so one bulk copy moves it into shared
// memory. Rows i >= I and columns j >= J are zero.
constexpr int FD_KC = 64;     // bytes of the reduction (row) dimension per chunk
constexpr int FD_MT = 128;    // database columns per MMA tile (the M dimension)
constexpr int FD_LIMBS = 5;   // bytes per residue
constexpr int FD_PLANE = FD_MT * FD_KC;             // 8192 bytes: one byte plane of a chunk
constexpr int FD_CHUNK = FD_LIMBS * FD_PLANE;       // 40960 bytes
// Packed chunks (q2 < 2^34, so byte 4 of a residue is below 4): planes 0..3 as
// above, then byte 4 at two bits per residue (2048 bytes): for every quad Q of
// four consecutive 16-byte groups of the unpacked plane (groups 4Q .. 4Q + 3 in
// core-matrix order), four u32 words P_w, w < 4, where bits 8b + 2k, 8b + 2k + 1
// of P_w hold byte 4w + b of group 4Q + k. Unpacking a group is then one shift
// and one mask per word: word w of group 4Q + k = (P_w >> 2k) & 0x03030303.
constexpr int FD_PACK4 = FD_PLANE / 4;                 // 2048 bytes
constexpr int FD_CHUNK_P4 = 4 * FD_PLANE + FD_PACK4;   // 34816 bytes

// One scan tile choice, the autotuner's search space. Every choice computes the
// same exact sums; they differ in speed only.
//  n_max  : selection columns per c-tile for batches (16, 24, 32 or 48); the
//           batch's 2*nq columns are spread evenly over ceil(2nq / n_max)
//           tiles, each padded to a multiple of 16 (of 8 for n_max = 24, whose
//           MMA operand is padded with zero rows to a multiple of 16). Tiles of
//           at most 24 columns hold two accumulator sets in TMEM, so the MMAs of
//           one column tile overlap the epilogue of the previous one.
//  stages : depth of the shared-memory ring of (database, selection) chunks.
//  order  : 0 walks units slot-major (the c-tiles of one slot run on
//           neighbouring SMs at the same time and share the slot's planes in
//           L2); 1 walks them tile-major (one c-tile over every slot, then the next).
// Zero fields take the built-in default (48 columns, 3 stages; 4 for one query).
struct FdTile {
  int n_max = 0, stages = 0, order = 0;
};

struct FdPlan {
  const uint8_t* planes = nullptr;
  int I = 0, J = 0, n = 0;  // rows, columns, ring degree
  int I_pad = 0, J_pad = 0;
  DevMod m{};
  int grid = 148;          // persistent CTAs (one per SM)
  int smem_max = 0;        // opt-in shared memory per block on this device
  bool packed4 = false;    // chunks in the packed layout (FD_CHUNK_P4 bytes each)
  int* err = nullptr;      // device word: nonzero after a bounded wait ran out
  // Test hook (via_server_set_scan_fault): when nonzero, the epilogue of every
  // CTA first waits on a barrier that nothing completes, bounded by this many
  // nanoseconds, so the scan's abort path runs and the error word is set.
  unsigned fault_wait_ns = 0;
  // Tuned tiles by batch size, sorted by batch. A scan of nq queries uses the
  // entry of the smallest tuned batch >= nq of the same kind (one query or a
  // batch), else the largest below it, else the default.
  std::vector<std::pair<int, FdTile>> tuned;
};

inline int fd_round_up(int v, int a) { return (v + a - 1) / a * a; }
size_t fd_planes_bytes(int I, int J, int n, bool packed4);
// The packed layout serves moduli below 2^34.
inline bool fd_packable(u64 q) { return q < (1ull << 34); }
bool fd_supported(int I, int n, u64 q);

// The tile a scan of nq queries runs with (tuned entry or default).
FdTile fd_tile_for(const FdPlan& p, int nq);
// Every tile the autotuner tries for nq queries (all valid on this device).
std::vector<FdTile> fd_tile_candidates(const FdPlan& p, int nq);
bool fd_tile_valid(const FdPlan& p, int nq, const FdTile& t);
// Records `t` as the tile for batches of nq (replacing an entry for nq).
void fd_set_tile(FdPlan& p, int nq, const FdTile& t);

struct FdTuneResult {
  FdTile tile;
  float ms = 0.f;
};
// Times every candidate tile for nq queries on the given buffers (their
// contents are irrelevant to the timing and are overwritten): one warm-up scan
// and `reps` timed scans each, with CUDA events on `st`. Returns the
// measurements in candidate order; the first entry is the default tile.
std::vector<FdTuneResult> fd_measure_tiles(const FdPlan& p, int nq, const u64* sel_eval, u64* out_eval,
                                           uint8_t* scratch, cudaStream_t st, int reps);

// Converts rows [i0, i0 + 16) of an eval-form database held as u64 [16][J][n]
// (`stage`, rows beyond I ignored) into the byte planes.
void fd_rows_to_planes(const u64* stage, int i0, const FdPlan& p, uint8_t* planes, cudaStream_t st);

// Raises the scan kernel's shared-memory limit on the current device to the
// device's opt-in maximum (once per device, before the first fd_scan there) and
// returns that maximum in bytes.
int fd_prepare_device();

// Scratch (bytes) that fd_scan needs for nq queries' split selection vectors,
// whichever candidate tile the scan runs with.
size_t fd_sel_bytes(const FdPlan& p, int nq);

// out_eval[b][j] = sum_i sel_eval[b][i] (.) db[i][j] for mask and body:
// sel_eval [nq][I][2][n], out_eval [nq][J][2][n], eval form mod q2. `force`
// overrides the tuned tile (it must be valid for nq).
void fd_scan(const FdPlan& p, const u64* sel_eval, u64* out_eval, int nq, uint8_t* scratch, cudaStream_t st,
             const FdTile* force = nullptr);

}  // namespace via
