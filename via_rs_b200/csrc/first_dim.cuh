#pragma once
#include "common.cuh"

namespace via {

// out_eval[j] = sum_i db[i][j] (.) sel_eval[i] for mask and body, eval domain at q2.
// db: [I][J][n]; sel_eval: I RLWEs (mask, body) [I][2][n]; out_eval: [J][2][n].
// `ntt` selects pointwise products (NTT-friendly q2) or negacyclic schoolbook.
// sel_split: scratch of I*2*n uint2; variant: column tile (0..first_dim_variants()-1).
void first_dim_eval(const u64* db, const u64* sel_eval, u64* out_eval, int I, int J, int n, const DevMod& m, bool ntt,
                    cudaStream_t st, uint2* sel_split, int variant);
// The same for nq queries sharing one pass over the database: sel_eval
// [nq][I][2][n], out_eval [nq][J][2][n], sel_split [nq][I][2][n] uint2.
void first_dim_eval_batch(const u64* db, const u64* sel_eval, u64* out_eval, int nq, int I, int J, int n,
                          const DevMod& m, bool ntt, cudaStream_t st, uint2* sel_split, int variant);
int first_dim_variants();
bool first_dim_split_ok(int I, int n, u64 q);

}  // namespace via
