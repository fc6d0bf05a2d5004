#pragma once
#include "common.cuh"

namespace via {

// out[j] = sum_i db[i][j] * sel[i] (negacyclic products, exact) for mask and
// body: db [I][J][n], sel [I][2][n], out [J][2][n], all coefficient form.
void first_dim_schoolbook(const u64* db, const u64* sel, u64* out, int I, int J, int n, const DevMod& m,
                          cudaStream_t st);

}  // namespace via
