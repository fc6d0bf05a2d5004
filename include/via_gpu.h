/*
 * via_gpu.h — C ABI of the B200 VIA server answer path.
 *
 * This library is a drop-in for the reference (roynalnaruto/via-rs) server API
 * `via_server::Server` (crates/via-server/src/answer.rs:423-603):
 *
 *   Server::setup(ServerConfig, &[RRec], p_mod)  -> via_server_setup
 *   Server::answer(&CompressedQuery)             -> via_server_answer
 *   drop(Server)                                 -> via_server_destroy
 *
 * plus the free kernel boundaries the reference names for a GPU build
 * (`first_dim`, crates/via-server/src/first_dim.rs:94; the eval-form gadget
 * product, crates/via-primitives/src/encryption/rlev.rs:259) as device-pointer
 * entry points for parity tests and micro-benchmarks.
 *
 * Conventions
 *  - Plain C99: opaque handles, caller-owned buffers of little-endian uint64_t
 *    residues, an int status. No CUDA or torch types cross the boundary; a
 *    stream is passed as `void*` (a cudaStream_t, or NULL for the default).
 *  - All ciphertext buffers use the reference's in-memory layout:
 *      poly   : nl limb arrays of n residues, limb 0 first
 *               (PolyRns, crates/via-primitives/src/algebra/ring/rns_element.rs:44-54);
 *               nl = 2 at q1 when q1 is a two-prime RNS basis, else 1.
 *      RLWE   : mask poly, then body poly.
 *      RLev   : L RLWE samples, samples[0] paired with the largest gadget entry
 *               (crates/via-primitives/src/encryption/types.rs:148-251).
 *      LWE    : MLWECiphertext<n1, 1> (crates/via-primitives/src/encryption/mlwe.rs:27-39)
 *               stored as its mask polynomial (nl*n1, coefficient i = masks[i])
 *               followed by the body (nl residues).
 *      query  : the CompressedQuery's LWEs in order (DMux bits MSB-first,
 *               CMux bits LSB-first, CRot bits LSB-first, L_QUERY levels each).
 *      answer : ModSwitchedCiphertext<n2> = mask (n2 residues mod q3) then
 *               body (n2 residues mod q4).
 *  - Status codes are the reference's ViaError discriminants + 1
 *    (crates/via-protocol/src/error.rs:20-64), then device-side codes.
 */
#ifndef VIA_GPU_H
#define VIA_GPU_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef enum via_status {
  VIA_OK = 0,
  VIA_ERR_SETUP_NOT_COMPLETE = 1,      /* ViaError::SetupNotComplete */
  VIA_ERR_INDEX_OUT_OF_RANGE = 2,      /* ViaError::IndexOutOfRange */
  VIA_ERR_QUERY_LENGTH_MISMATCH = 3,   /* ViaError::QueryLengthMismatch */
  VIA_ERR_BUFFER_TOO_SHORT = 4,        /* ViaError::BufferTooShort */
  VIA_ERR_UNKNOWN_FORMAT_TAG = 5,      /* ViaError::UnknownFormatTag */
  VIA_ERR_INVALID_PRG_SEED = 6,        /* ViaError::InvalidPrgSeed */
  VIA_ERR_DIM_MISMATCH = 7,            /* ViaError::DimMismatch */
  VIA_ERR_INVALID_ARGUMENT = 100,      /* null handle/pointer, unsupported parameter */
  VIA_ERR_OUT_OF_MEMORY = 101,         /* device allocation or HBM budget exhausted */
  VIA_ERR_CUDA = 102,                  /* a CUDA runtime call failed */
  VIA_ERR_TIMEOUT = 103,               /* a bounded wait expired */
  VIA_ERR_BUSY = 104                   /* serving queue full; retry later */
} via_status;

/*
 * Runtime mirror of the reference's const-generic preset + PIRParams
 * (crates/via-protocol/src/params.rs:59-125, presets.rs:204-258) and the
 * server's DB dimensions (PublicParams.num_rows/num_cols) and record degree
 * N_REC (answer.rs:423-434).
 */
typedef struct via_params {
  uint32_t n1;        /* large ring degree (power of two) */
  uint32_t n2;        /* small ring degree, n1 = d * n2 */
  uint32_t n_rec;     /* record degree: n2 for VIA-C, n3 for VIA-B */
  uint32_t reserved0;
  uint64_t num_rows;  /* I (power of two) */
  uint64_t num_cols;  /* J (power of two) */
  uint64_t q1_0;      /* q1 = q1_0 * q1_1 (two-prime RNS) ... */
  uint64_t q1_1;      /* ... or q1 = q1_0 when q1_1 == 0 */
  uint64_t q2, q3, q4, p;
  uint64_t b_dmux;    /* gadget_base_1 (DMux @ q1) */
  uint64_t b_cmux;    /* gadget_base_2 (CMux / CRot @ q2) */
  uint64_t ck_base;   /* cascade + conversion-key gadget base */
  uint64_t b_rsk;     /* ring-switch gadget base */
  uint32_t l_query;   /* L_QUERY: LWEs per query bit = RGSW gadget depth */
  uint32_t l_ck;      /* L_CK: cascade / conversion-key depth */
  uint32_t l_rsk;     /* L_RSK: ring-switch key depth */
  uint32_t reserved1;
} via_params;

/* Record encodings accepted by via_server_setup. */
typedef enum via_record_format {
  VIA_RECORDS_U64 = 0,    /* n_rec uint64_t coefficients per record (reference RRec layout) */
  VIA_RECORDS_NIBBLE = 1  /* n_rec/2 bytes per record, two 4-bit coefficients per byte,
                             low nibble first (requires p <= 16) */
} via_record_format;

/* The client's public keys (reference PublicParams, crates/via-protocol/src/wire/keys.rs:29-108). */
typedef struct via_public_keys {
  const uint64_t* cascade_key; /* LWE->RLWE cascade key: for k = 1..log2 n1, RANK_IN = n1>>(k-1)
                                  RLevs of L_CK samples at degree 2^k over q1 (prim/conversion/cascade.rs) */
  const uint64_t* conv_key;    /* RLev_{S1}(S1^2): L_CK samples at (q1, n1) */
  const uint64_t* rsk;         /* ring-switch key: d RLevs of L_RSK samples at (q3, n2) */
} via_public_keys;

typedef struct via_server via_server;

/* Buffer sizes in uint64_t units. */
uint64_t via_lwe_len(const via_params* p);
uint64_t via_query_len(const via_params* p);          /* number of LWEs in a query */
uint64_t via_cascade_key_len(const via_params* p);
uint64_t via_conv_key_len(const via_params* p);
uint64_t via_rsk_len(const via_params* p);

/*
 * Server::setup (answer.rs:486-528): encodes the records into the I x J cell
 * matrix (setup_db.rs:39-75), lifts them to q2 and forward-transforms them on
 * the device once (prepared_db.rs:57-85), and uploads the eval-form public keys
 * (prepared_keys.rs:69-79). Fewer records than capacity are zero-padded; more
 * is VIA_ERR_DIM_MISMATCH. Uses the calling thread's current CUDA device.
 */
via_status via_server_setup(const via_params* params, const via_public_keys* keys, const void* records,
                            uint64_t n_records, via_record_format format, via_server** out);

/*
 * A second server handle over the prepared database of `base` (no copy) with
 * another record degree: n_rec = n2 for VIA-C, or a VIA-B n3 dividing n2. The
 * database is a grid of I x J cells of n1 plaintext coefficients; a server
 * reads it as records of degree n_rec, record k*I*J + i*J + j being
 * coefficients d*c + k (c < n_rec, d = n1 / n_rec) of cell (i, j), which is how
 * setup_db (setup_db.rs:39-75) places records of that degree. So one copy of a
 * database in HBM serves VIA-C queries and VIA-B batches of any T side by side.
 * `keys` may be the base's or another client's. The cells stay alive while
 * any handle over them does; destroy handles in any order. The reference
 * builds one Server per record degree, each with its own PreparedDb.
 */
via_status via_server_view(via_server* base, uint32_t n_rec, const via_public_keys* keys, via_server** out);

/*
 * Server::answer (answer.rs:534-554): steps 1-7 on the device for one query.
 * out_mask: n2 residues mod q3; out_body: n2 residues mod q4. Host buffers.
 */
via_status via_server_answer(via_server* s, const uint64_t* query, uint64_t n_lwe, uint64_t* out_mask,
                             uint64_t* out_body);

/*
 * The same answer on device buffers, enqueued on `stream` without a host
 * synchronisation: `query` (n_lwe LWEs), `out_mask`, `out_body` are device
 * pointers. Answers on one handle are serialised (it owns one workspace).
 */
via_status via_server_answer_dev(via_server* s, const uint64_t* query, uint64_t n_lwe, uint64_t* out_mask,
                                 uint64_t* out_body, void* stream);

/*
 * Many independent VIA-C queries answered together: one pass over the
 * database serves the whole batch (FirstDim is linear, so each column sum is
 * the same as answering alone), and every other step runs on all queries'
 * ciphertexts at once. `queries` holds n_queries queries back to back;
 * out_masks / out_bodies receive n_queries answers of n2 residues each. The
 * results equal n_queries calls of via_server_answer. Host buffers.
 */
via_status via_server_answer_many(via_server* s, const uint64_t* queries, uint64_t n_queries, uint64_t n_lwe,
                                  uint64_t* out_masks, uint64_t* out_bodies);

/* The same on device buffers, enqueued on `stream`. */
via_status via_server_answer_many_dev(via_server* s, const uint64_t* queries, uint64_t n_queries, uint64_t n_lwe,
                                      uint64_t* out_masks, uint64_t* out_bodies, void* stream);

/* Sizes the per-handle workspace for batches of up to max_queries (it also
 * grows on demand). */
via_status via_server_reserve(via_server* s, uint64_t max_queries);

void via_server_destroy(via_server* s);

/* Message for the last failing call on this thread ("" if none). */
const char* via_last_error(void);

/*
 * FirstDim (first_dim.rs:94-184) on device buffers: `switched` holds I RLWEs at
 * (q2, n1) in coefficient form; `out` receives the J column RLWEs. The server's
 * prepared database is the other operand.
 */
via_status via_first_dim_dev(via_server* s, const uint64_t* switched, uint64_t* out, void* stream);

/*
 * The FirstDim scan kernel alone, on eval-form operands: `sel_eval` holds the I
 * selection RLWEs already transformed, `out_eval` receives the J column sums
 * untransformed. For timing the database scan in isolation.
 */
via_status via_first_dim_scan_dev(via_server* s, const uint64_t* sel_eval, uint64_t* out_eval, void* stream);

/*
 * The server's own negacyclic transform at (q2, n1), in place on `count`
 * polynomials of n1 residues: forward (inverse = 0) gives the eval form the
 * scan entry points above take and return, inverse (inverse = 1) brings their
 * outputs back to coefficients. The order of eval slots is this library's
 * (first_dim.rs:94-184 only observes coefficient-form results). Servers whose
 * q2 has no NTT use coefficients as their eval form: the call is a no-op.
 * Enqueued on `stream`.
 */
via_status via_server_transform_q2_dev(via_server* s, uint64_t* data, uint64_t count, int inverse, void* stream);

/*
 * The scans of n_queries independent queries in one pass over the database
 * (the T first_dim calls of answer_batch, srv/batch.rs:139-150, sharing the
 * scan): `sel_eval` holds [n_queries][I][2][n1] eval-form selection RLWEs,
 * `out_eval` receives [n_queries][J][2][n1]. Allocates its scratch per call.
 */
via_status via_first_dim_scan_many_dev(via_server* s, const uint64_t* sel_eval, uint64_t n_queries,
                                       uint64_t* out_eval, void* stream);

/*
 * Scan autotuner. The FirstDim scan (`first_dim`, first_dim.rs:94-184, run as a
 * tensor-core integer GEMM) has a tile space: selection columns per tile for
 * batches, the depth of its shared-memory ring, and the order its persistent
 * CTAs walk the (slot, column-tile) units in. Every tile gives the same exact
 * result. via_server_autotune times every candidate tile for each listed batch
 * size on this server's database (CUDA events, one warm-up and three timed
 * scans each, in two passes over the candidates) and keeps the candidate whose
 * faster pass is fastest; scans of other batch sizes use the entry
 * of the nearest tuned size above (else below) of the same kind (one query, or
 * a batch). With a cache_path, entries measured before for the same device,
 * ring degree, grid and modulus are read from that file instead of measured,
 * and new measurements are appended to it. Answer graphs captured before the
 * call are re-captured on next use. Servers on non-NTT rings have no tiles:
 * their entries report 0 candidates. `out` (may be NULL) receives one entry
 * per batch size. No counterpart in the reference, whose FirstDim is a
 * threaded CPU loop.
 */
typedef struct via_scan_tile {
  uint32_t n_max;    /* selection columns per tile for batches: 16, 24, 32 or 48; 0 = default (48) */
  uint32_t stages;   /* shared-memory ring depth, 2..6; 0 = default (3; 4 for one query) */
  uint32_t order;    /* 0: slot-major units, 1: tile-major units (batches only) */
  uint32_t reserved;
} via_scan_tile;

typedef struct via_scan_tuning {
  uint32_t batch;       /* queries per scan */
  via_scan_tile tile;   /* the tile kept */
  float ms;             /* its scan time in milliseconds */
  float default_ms;     /* the default tile's scan time */
  uint32_t candidates;  /* tiles measured; 0 when read from the cache file */
  uint32_t reserved;
} via_scan_tuning;

via_status via_server_autotune(via_server* s, const uint32_t* batch_sizes, uint64_t count, const char* cache_path,
                               via_scan_tuning* out);
/* Sets (tile != NULL) or clears the tile used for scans of `batch` queries. */
via_status via_server_set_scan_tile(via_server* s, uint32_t batch, const via_scan_tile* tile);
/* The candidate tiles for `batch` queries (the default first); returns their
 * number and writes up to `cap` of them to `out` (may be NULL). */
uint64_t via_scan_tile_candidates(via_server* s, uint32_t batch, via_scan_tile* out, uint64_t cap);

/*
 * Test hook for the scan's bounded device waits. With wait_us > 0 (at most
 * 100000), every later FirstDim scan on this handle first makes its epilogue
 * wait on a barrier that nothing completes, for wait_us microseconds; the wait
 * runs out, the CTAs abort (after their copies and MMAs in flight have landed)
 * and set the handle's error word, so the synchronous calls and service
 * requests report VIA_ERR_TIMEOUT, as after a real stall. wait_us = 0 turns the
 * hook off and clears the error word. Returns VIA_ERR_INVALID_ARGUMENT for
 * servers on non-NTT rings (their scan has no waits). The reference has no
 * device and no counterpart; its error contract is proto/error.rs:20-64.
 */
via_status via_server_set_scan_fault(via_server* s, uint32_t wait_us);

/*
 * Runs the answer up to `stage` and copies that stage's output, in coefficient
 * form, to the host buffer `out` (for stage-by-stage parity checks):
 *   1 cascade RLWEs [n_lwe][2][nl][n1]      (query_decomp.rs:76-78)
 *   2 query RGSWs at q1 [bits][2L][2][nl][n1] (query_decomp.rs:81-85)
 *   3 DMux outputs [I][2][nl][n1]            (answer.rs:181-191)
 *   4 mod-switched rows at q2 [I][2][n1]     (answer.rs:194-199)
 *   5 FirstDim columns [J][2][n1]            (answer.rs:204-205)
 *   6 CMux output [2][n1]                    (answer.rs:208-215)
 *   7 CRot output [2][n1]                    (answer.rs:218-225)
 */
via_status via_debug_stage(via_server* s, const uint64_t* query, uint64_t n_lwe, int stage, uint64_t* out,
                           uint64_t out_len);

/*
 * Server::answer_batch (VIA-B, crates/via-server/src/batch.rs:72-163): the
 * server must have been set up with n_rec < n2; the batch size is then
 * T = n2 / n_rec (the record-fit boundary T * n_rec = n2). `queries` holds T
 * queries of n_lwe LWEs each, back to back (layout of via_server_answer); the
 * single answer (n2 mask residues at q3, n2 body residues at q4) packs the T
 * records, record t at plaintext slots t + (n2 / n_rec) * k. The T queries share
 * one database scan, then the T CRot outputs are repacked (repack.rs) with the
 * cascade key's last log2(n1 / n_rec) steps switched to q2, and RespComp runs
 * once. VIA_ERR_DIM_MISMATCH when n_queries != T or the server is VIA-C only.
 */
via_status via_server_answer_batch(via_server* s, const uint64_t* queries, uint64_t n_queries, uint64_t n_lwe,
                                   uint64_t* out_mask, uint64_t* out_body);
/* The same on device buffers, enqueued on `stream` (`queries` is read in place,
 * so it must stay valid until the stream reaches the end of this work). Both
 * entry points run batches of more than 64 queries (T = 256) through their
 * prefix in chunks of 64, each chunk sharing one database scan. */
via_status via_server_answer_batch_dev(via_server* s, const uint64_t* queries, uint64_t n_queries, uint64_t n_lwe,
                                       uint64_t* out_mask, uint64_t* out_body, void* stream);

/*
 * Serving: a continuous-batching answer service over one server handle (the
 * request loop the reference leaves to its caller). Requests are queued on
 * the host; a worker thread keeps `lanes` batches in flight, each on its own
 * stream and workspace, and whenever a lane frees up it takes every pending
 * request up to the lane's capacity (one database scan per batch). The
 * capacity is the largest batch whose workspace fits hbm_budget / lanes, capped
 * by max_batch; requests beyond it wait for a free lane. A VIA-C server serves
 * single queries; a VIA-B server (n_rec < n2) serves groups of T = n2 / n_rec
 * queries, one answer per group; a group larger than a lane's workspace runs
 * alone, its prefix in chunks. Results do not depend on how requests are
 * batched. Every wait is bounded; no host thread blocks inside the driver.
 * Services over views of one database (via_server_view) serve VIA-C queries
 * and VIA-B batches of several T from a single copy of the database.
 */
typedef struct via_service via_service;

typedef struct {
  uint32_t lanes;       /* batches in flight; 0 -> 2 */
  uint32_t max_batch;   /* requests per batch; 0 -> 64 */
  uint64_t hbm_budget;  /* device bytes for all lanes' workspaces; 0 -> max_batch decides */
  uint32_t max_pending; /* queued requests before submit returns VIA_ERR_BUSY; 0 -> 2^20 */
  uint32_t warm;        /* nonzero: capture every batch size's answer graph at creation */
  uint32_t autotune;    /* nonzero: run the scan autotuner (via_server_autotune) at creation
                           for the batch sizes 1, 2, 4, ... up to the lane capacity */
  const char* tune_cache; /* the autotuner's cache file, or NULL */
} via_service_config;

typedef struct {
  uint64_t submitted, completed, failed, batches, units;
  uint32_t lanes, batch_cap;
  uint32_t max_in_flight; /* most batches seen on the GPU at once */
  uint32_t reserved;
  double p50_ms, p99_ms;  /* submit-to-completion latency of completed requests */
  double mean_batch;      /* requests per launched batch */
  double answers_per_s;   /* completed requests / (last completion - first submit) */
} via_service_stats;

via_status via_service_create(via_server* s, const via_service_config* cfg, via_service** out);
/* Device bytes of one lane's workspace for batches of up to max_queries queries
 * (for sizing hbm_budget); 0 on a null handle. */
uint64_t via_server_workspace_bytes(via_server* s, uint64_t max_queries);
/* Queues one request: a query of n_lwe LWEs (VIA-C) or T such queries back to
 * back (VIA-B); the buffer is copied. Returns a ticket. */
via_status via_service_submit(via_service* v, const uint64_t* query, uint64_t n_lwe, uint64_t* ticket);
/* Non-blocking: *done = 1 and the answer (n2 + n2 residues) once finished; the
 * ticket is then released. */
via_status via_service_poll(via_service* v, uint64_t ticket, uint64_t* out_mask, uint64_t* out_body, int* done);
/* Waits up to timeout_ms (VIA_ERR_TIMEOUT after that, the ticket stays valid). */
via_status via_service_wait(via_service* v, uint64_t ticket, uint64_t* out_mask, uint64_t* out_body,
                            uint32_t timeout_ms);
via_status via_service_stats_get(via_service* v, via_service_stats* out);
/* Zeroes the counters and latency record (requests in flight still complete). */
via_status via_service_stats_reset(via_service* v);
/* Submit-to-completion latencies (milliseconds) of the requests completed since
 * creation or the last stats reset, in completion order: returns their number
 * and writes up to `cap` of them to `out` (may be NULL). */
uint64_t via_service_latencies(via_service* v, double* out, uint64_t cap);
/* The autotuner's choices made at creation (cfg.autotune): returns their
 * number and writes up to `cap` entries to `out` (may be NULL). */
uint64_t via_service_tuning(via_service* v, via_scan_tuning* out, uint64_t cap);
/* Finishes the batches on the GPU, drops queued requests, frees the lanes. */
void via_service_destroy(via_service* v);

/*
 * Query wire formats (via-protocol/src/wire/format.rs:93-190). A wire query is
 * n_lwe packets, one per LWE, each led by the format tag:
 *   0x00 Uncompressed : [0x00][count u64 LE = nl*(n1+1)][the LWE's u64s, LE]
 *   0x01 PrgCompressed: [0x01][seed, 32 bytes][count u64 LE = nl][the body's u64s, LE]
 * A compressed packet's mask is regenerated as Shake256Prg(seed).uniform_below(q_l),
 * row-major, one draw per limb, limb 0 first (format.rs:20-27); the device
 * computes the PRG blocks in parallel. Errors: VIA_ERR_UNKNOWN_FORMAT_TAG,
 * VIA_ERR_BUFFER_TOO_SHORT (truncated or too few packets),
 * VIA_ERR_QUERY_LENGTH_MISMATCH (bytes after the last packet),
 * VIA_ERR_DIM_MISMATCH (a packet's count does not match the parameters).
 */
via_status via_query_from_wire(via_server* s, const uint8_t* wire, uint64_t len, uint64_t* out_query,
                               uint64_t out_len);
/* Decodes a wire query on the device and answers it (host answer buffers). */
via_status via_server_answer_wire(via_server* s, const uint8_t* wire, uint64_t len, uint64_t* out_mask,
                                  uint64_t* out_body);

/*
 * The FirstDim scan of via_first_dim_scan_dev for callers that cannot allocate
 * device memory: a host whose device memory is owned by another runtime's
 * allocator or a fixed pool (cudaMalloc there would fail or bypass its
 * accounting), or a latency-critical path that must not enter the allocator,
 * which can synchronize the device. It allocates nothing: its scratch (the
 * split selection vectors) is a static 8 MiB device array that the library
 * holds on every device until exit. It requires 16 * I_pad * n1 <= 2^23 bytes,
 * I_pad = num_rows rounded up to 64 (I <= 256 at n1 = 2048, I <= 128 at
 * n1 = 4096), and returns VIA_ERR_INVALID_ARGUMENT above that; servers whose
 * q2 has no NTT (schoolbook rings) use no scratch and have no limit. Call it
 * with the server's device current (else VIA_ERR_INVALID_ARGUMENT). The first
 * call on a device looks up the array's device address; make it before any
 * stream capture. Calls share the array, which keeps the last call's contents:
 * calls whose work overlaps on the GPU race on it. Like via_first_dim_scan_dev
 * it returns once the scan is enqueued. This entry point has no counterpart in
 * the reference.
 */
via_status via_first_dim_scan_static(via_server* s, const uint64_t* sel_eval, uint64_t* out_eval, void* stream);

/*
 * Primitive operations on caller device buffers, over any NTT-friendly ring
 * (each prime below 2^50 and = 1 mod 2n; n a power of two in 2..4096). They run
 * the answer path's kernels on the reference's own operations, for parity
 * tests and the kernel micro-benchmarks. Layouts are the reference's (limb 0
 * first; RLWE = mask then body; RGSW = neg_s_m RLev then m RLev, L samples
 * each, sample 0 paired with the largest gadget entry). Every call is
 * enqueued on `stream`; the external product and key switch return after
 * their work has finished (they reuse a per-device scratch buffer).
 */
typedef struct via_ring_desc {
  uint32_t n;     /* degree */
  uint32_t nl;    /* 1, or 2 for a two-prime RNS modulus q[0] * q[1] */
  uint64_t q[2];
} via_ring_desc;

/* In-place negacyclic NTT of `count` ring elements [count][nl][n]: the
 * reference's cooley_tukey_dit_forward / cooley_tukey_dif_inverse
 * (algebra/ring/ntt.rs:305-399), with its root (the primitive 2n-th root from
 * the smallest base, ntt.rs:150-198) and bit-reversed evaluation order, so
 * the eval form equals the reference's. Outputs are canonical residues. */
via_status via_ntt_forward_dev(const via_ring_desc* ring, uint64_t* data, uint64_t count, void* stream);
via_status via_ntt_inverse_dev(const via_ring_desc* ring, uint64_t* data, uint64_t count, void* stream);

/* out[c] = rgsw[c] (x) rlwe[c] (encryption/rgsw.rs:108-121) for `count` pairs,
 * coefficient form, one gadget (base, levels) for both halves of the RGSW:
 * rgsw [count][2*levels][2][nl][n], rlwe and out [count][2][nl][n]. */
via_status via_external_product_dev(const via_ring_desc* ring, uint64_t base, uint32_t levels, const uint64_t* rgsw,
                                    const uint64_t* rlwe, uint64_t count, uint64_t* out, void* stream);

/* out[c] = key_switch(key, X^shifts[c] * rlwe[c]) (encryption/keyswitch.rs:99-102
 * after the monomial rotation of algebra/ring/element.rs:328, shift taken mod
 * 2n): key is one RLev of `levels` samples [levels][2][nl][n] in coefficient
 * form shared by all; rlwe and out [count][2][nl][n]. */
via_status via_key_switch_dev(const via_ring_desc* ring, uint64_t base, uint32_t levels, const uint64_t* key,
                              const uint64_t* rlwe, const uint64_t* shifts, uint64_t count, uint64_t* out,
                              void* stream);

/*
 * The client side on the device (crates/via-client/src), for load generation at
 * serving rates and for clients holding many queries. The client's secret keys
 * come from its keygen (cli/client.rs:89-180): sk1 is nl * n1 residues at q1
 * (limb 0 first), sk2 is n2 residues at q3. err_kind 0 samples ternary errors,
 * 1 bounded-uniform errors in [-err_bound, err_bound] (distribution.rs:88-118).
 */
typedef struct via_client via_client;
via_status via_client_create(const via_params* params, const uint64_t* sk1, const uint64_t* sk2, uint32_t err_kind,
                             uint32_t err_bound, via_client** out);
void via_client_destroy(via_client* c);

/* Client::query (cli/query.rs:75-130) for `count` indices: query k is drawn from
 * Shake256Prg(seeds + k * seed_len) (seed_len in 1..64 bytes), exactly as the
 * reference client would draw it from that PRG. Each query has via_query_len
 * LWEs (d = n1 / n_rec selects the CRot bits) in the via_server_answer layout;
 * `out` (host) receives count queries back to back. The PRG blocks are computed
 * in parallel, one warp walks each query's rejection-sampled stream, and the
 * inner products run one CTA per LWE. VIA_ERR_INDEX_OUT_OF_RANGE for an index
 * >= d * I * J. */
via_status via_client_queries(via_client* c, const uint64_t* indices, uint64_t count, const uint8_t* seeds,
                              uint32_t seed_len, uint64_t* out);
/* The same into device memory, enqueued on `stream`; returns after the work is done. */
via_status via_client_queries_dev(via_client* c, const uint64_t* indices, uint64_t count, const uint8_t* seeds,
                                  uint32_t seed_len, uint64_t* out, void* stream);
/* Client::recover for `count` answers (decrypt_asymmetric, encryption/rlwe.rs:187-240):
 * masks and bodies [count][n2] (host), out [count][n2] plaintext coefficients mod p.
 * VIA-B answers hold record t at coefficients t + T * k (recover_batch, cli/batch.rs:35-58). */
via_status via_client_recover(via_client* c, const uint64_t* masks, const uint64_t* bodies, uint64_t count,
                              uint64_t* out);

/* The gadget decomposition the kernels run (gadget.rs:115-190: centred lift,
 * round(|c| B^L / Q), balanced base-B digits LSB-first), evaluated on the host
 * for `count` coefficients given as residues (nl per coefficient; q1 = 0 for a
 * single modulus). out: count * levels digits. No device work: it checks the
 * exact scaling against the reference on machines without a GPU. */
via_status via_gadget_digits_host(uint64_t q0, uint64_t q1, uint64_t base, uint32_t levels, const uint64_t* coeffs,
                                  uint64_t count, int64_t* out);

/* Number of kernels this library has launched since it was loaded. */
uint64_t via_kernel_launches(void);

#ifdef __cplusplus
}
#endif

#endif /* VIA_GPU_H */
