// Host side of the bulk-copy block dot (fm_blockdot.cu).
#pragma once
#include <cuda_runtime.h>
#include <stddef.h>

namespace fm {

// Bytes of per-CTA partial sums the bulk block dot needs for this shape; 0 when it does not take the shape
// (the caller then uses k_blockdot_mma).  rbytes / ybytes: bytes of one real part of the basis / block
// vectors (4 or 8); nact: active right-hand sides; sms: persistent CTAs (one per SM).
size_t blockdot_bulk_part_bytes(int rbytes, int ybytes, int S, long long M, int nb, int nact, int K, int sms);

// D[b][k*S + t] = sum_e conj(X_k[b][e]) * Y_t[b][e] for the active right-hand sides b, into out[b*K*S + ...].
// U: K basis vectors, Y: S block vectors, both [vector][b][M].  counter[b] must be zero (it is left zero).
// A pipeline wait that timed out writes a non-zero code to *err.
cudaError_t launch_blockdot_bulk(int rbytes, int ybytes, int S, long long M, int nb, int nact, int K, const void* U,
                                 const void* Y, double2* part, size_t part_bytes, double2* out, unsigned* counter,
                                 const int* act, int* err, int sms, cudaStream_t st);

}  // namespace fm
