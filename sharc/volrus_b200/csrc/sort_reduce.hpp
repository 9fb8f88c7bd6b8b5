// Deterministic scatter-add by stable radix sort + segmented sum (sort_reduce.cu).
#pragma once
#include "vlr_host.hpp"

namespace vlr {

// Scratch bytes needed by sort_reduce for n pairs.
size_t sort_reduce_scratch_bytes(int n);
// out[k] = sum of vals[i] over keys[i] == k, summed in input order, for
// k < n_out (out is zeroed first; keys >= n_out are dropped).  keys < key_limit.
// keys and vals are clobbered.  Enqueued on the context stream.
int sort_reduce(vlr_ctx* ctx, unsigned* keys, float* vals, int n, unsigned key_limit, float* out, unsigned n_out,
                void* scratch);
// Stable LSD radix sort of (key, 32-bit payload) pairs by key (keys <=
// key_limit), enqueued on the context stream.  scratch holds
// sort_reduce_scratch_bytes(n); the sorted pairs end in either the input
// arrays or the scratch, as *keys_out / *vals_out report.
int radix_sort_pairs(vlr_ctx* ctx, unsigned* keys, unsigned* vals, int n, unsigned key_limit, void* scratch,
                     unsigned** keys_out, unsigned** vals_out);

}  // namespace vlr
