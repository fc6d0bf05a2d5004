// The device-resident server: parameters, NTT tables, prepared database and
// eval-form keys (crates/via-server/src/{answer,prepared_db,prepared_keys}.rs).
#pragma once
#include <memory>
#include <mutex>
#include <shared_mutex>
#include <string>
#include <vector>

#include "../../include/via_gpu.h"
#include "common.cuh"
#include "fd_tc.cuh"
#include "ntt.cuh"

namespace via {

// A ring as the kernels see it: degree, limb count and per-limb modulus/tables.
struct DevRing {
  int n = 0;
  int nl = 1;
  DevMod m[2];
  NttTable t[2];  // valid iff ntt
  bool ntt = false;
  u64 q0inv_mod_q1 = 0, q0inv_shoup = 0;  // CRT constants when nl == 2
  __host__ __device__ u128 Q() const { return nl == 1 ? (u128)m[0].q : (u128)m[0].q * m[1].q; }
  size_t size() const { return (size_t)nl * n; }
};

// Device buffer with RAII.
struct DevBuf {
  u64* p = nullptr;
  size_t n = 0;
  DevBuf() = default;
  explicit DevBuf(size_t count) { alloc(count); }
  void alloc(size_t count);
  void free();
  ~DevBuf() { free(); }
  DevBuf(const DevBuf&) = delete;
  DevBuf& operator=(const DevBuf&) = delete;
};

struct Workspace;  // per-query scratch (pipeline.cu)
struct WorkspaceDeleter {
  void operator()(Workspace* w) const;
};

struct Server {
  via_params prm{};
  int device = 0;
  cudaStream_t stream = nullptr;
  // Rings: q1 at n1 (1 or 2 limbs), q2 at n1, q3 at n1 and n2, q4 at n2.
  DevRing r1, r2, r3n1, r3, r4;
  std::vector<NttTableHost> tables;  // owners
  // Prepared database. NTT-friendly q2: byte planes for the tensor-core scan
  // (fd_tc.cuh layout) in `planes`, described by `fd`. Otherwise (schoolbook
  // rings): [I][J][n1] u64 residues in `db`.
  // Shared with the views of this database (via_server_view).
  std::shared_ptr<DevBuf> db;
  std::shared_ptr<DevBuf> planes;
  FdPlan fd;
  DevBuf fd_err;  // one device word the scan sets when a bounded wait runs out
  // Eval-form keys (crates/via-server/src/prepared_keys.rs:69-79).
  DevBuf cascade_eval;  // include/via_gpu.h cascade layout, each segment transformed
  DevBuf cascade_eval_d;  // the same residues as exact doubles (q1 primes below 2^44), for the double-precision MAC
  DevBuf conv_eval;     // L_CK samples at (q1, n1)
  DevBuf rsk_eval;      // d RLevs at (q3, n2)
  // VIA-B repack keys (n_rec < n2): the cascade steps of output degree 2 n_rec .. n1,
  // every sample switched q1 -> q2 and in eval form at q2; level l starts at repack_off[l].
  DevBuf repack_eval;
  std::vector<size_t> repack_off;
  std::unique_ptr<Workspace, WorkspaceDeleter> ws;
  std::mutex mu;  // one in-flight answer per handle (the workspace is shared)
  int plan_gen = 0;  // bumped when the scan tiles change; captured graphs of older plans are dropped
  // Guards fd.tuned and plan_gen: the autotuner holds it exclusively, service
  // workers (which do not take `mu`) hold it shared while they enqueue a batch.
  std::shared_mutex plan_mu;
  bool tensor_fd() const { return fd.planes != nullptr; }
  ~Server();
};

// Shared helpers.
void set_last_error(const std::string& m);  // the message via_last_error() returns
void validate_params(const via_params& p);
u64 lwe_len(const via_params& p);
u64 query_lwes(const via_params& p);
u64 cascade_key_len(const via_params& p);
u64 conv_key_len(const via_params& p);
u64 rsk_len(const via_params& p);
int ilog2(u64 v);
u64 h_inv(u64 a, u64 m);  // a^-1 mod m, 0 if not invertible

// Pipeline entry points (pipeline.cu).
constexpr int STOP_AFTER_CROT = -1;  // answer_device_stages: leave the CRot outputs in the workspace
// VIA-B batch size T = n2 / n_rec (the record-fit boundary); 1 for VIA-C servers.
inline int via_b_batch(const via_params& p) { return (int)(p.n2 / p.n_rec); }
// Queries per workspace pass of the synchronous VIA-B entry points: larger
// batches run their prefix in chunks of this many queries.
constexpr int VIA_B_CHUNK = 64;
void derive_repack_keys(Server& s);
void answer_batch_device(Server& s, const u64* d_queries, u64* d_mask, u64* d_body, cudaStream_t st);
void workspace_create(Server& s, int bmax);
std::unique_ptr<Workspace, WorkspaceDeleter> workspace_make(Server& s, int bmax);
size_t workspace_bytes(Server& s, int bmax);  // device bytes of a workspace for bmax queries
u64* ws_query(Workspace& w);
u64* ws_answer_mask(Workspace& w);
u64* ws_answer_body(Workspace& w);
void answer_graph(Server& s, Workspace& w, int nq, cudaStream_t st);
void answer_batch_device(Server& s, Workspace& w, const u64* d_queries, int groups, u64* d_mask, u64* d_body,
                         cudaStream_t st);
int workspace_batch(Server& s);
void workspace_destroy(Server& s);
uint8_t* workspace_sel_bytes(Server& s);
// FirstDim of nq queries: sel_eval [nq][I][2][n1] -> out_eval [nq][J][2][n1] (eval at q2).
void first_dim_queries(Server& s, const u64* sel_eval, u64* out_eval, int nq, uint8_t* scratch, cudaStream_t st);
std::vector<FdTuneResult> workspace_measure_tiles(Server& s, Workspace& w, int nq, int reps);
// The scan autotuner (server.cu): measures (or reads from the cache file) the
// fastest tile for every batch size on workspace w, records it in s.fd and
// invalidates captured graphs. The caller holds s.mu.
void autotune_scan(Server& s, Workspace& w, const std::vector<int>& sizes, const char* cache_path,
                   std::vector<via_scan_tuning>* out);
u64* workspace_query(Server& s);
u64* workspace_answer_mask(Server& s);
u64* workspace_answer_body(Server& s);
void answer_graph(Server& s, int nq, cudaStream_t st);
void answer_device(Server& s, const u64* d_query, u64* d_mask, u64* d_body, cudaStream_t st);
void answer_device_stages(Server& s, const u64* d_query, int nq, u64* d_mask, u64* d_body, cudaStream_t st,
                          int stop_stage, u64* dump);

}  // namespace via

struct via_server : via::Server {};
