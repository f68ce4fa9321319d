// Compressed nonzero list of the MPO mixing step, built cooperatively by one CTA in shared memory.
//
// The mix computes out[n, s'] = sum_{m,s} W[m + DL (n + DR (s + S s'))] in[m, s] for every (a', b) point.
// MPOs of spin chains are mostly zeros (the merged two-site Ising MPO keeps ~20% of its entries), so each CTA
// first lists, per output o = n*S + s', the nonzero (input slot m*S + s, weight) pairs, then every thread
// runs the short lists instead of the dense DL*S x DR*S block.
#pragma once
#include "heff_common.cuh"

namespace heff {

__device__ __forceinline__ bool wl_nz(double w) { return w != 0.0; }
__device__ __forceinline__ bool wl_nz(double2 w) { return w.x != 0.0 || w.y != 0.0; }

// Shared-memory footprint of the list for the given MPO block (bytes, 16-byte aligned pieces).
__host__ __device__ inline size_t wlist_bytes(int DL, int DR, int S, size_t wsize) {
    const size_t no = (size_t)DR * S, nnz = (size_t)DL * DR * S * S;
    auto         al = [](size_t b) { return (b + 15) / 16 * 16; };
    return al(4 * (no + 1)) + al(2 * nnz) + al(wsize * nnz);
}

template<class T>
__device__ void build_wlist(const T *sW, int DL, int DR, int S, unsigned char *mem, int *&off, short *&idx, T *&wv) {
    const int    NO  = DR * S;
    const size_t nnz = (size_t)DL * DR * S * S;
    auto         al  = [](size_t b) { return (b + 15) / 16 * 16; };
    off              = reinterpret_cast<int *>(mem);
    idx              = reinterpret_cast<short *>(mem + al(4 * (NO + 1)));
    wv               = reinterpret_cast<T *>(mem + al(4 * (NO + 1)) + al(2 * nnz));
    for(int o = threadIdx.x; o < NO; o += blockDim.x) {
        const int n = o / S, sp = o % S;
        int       c = 0;
        for(int s = 0; s < S; s++)
            for(int m = 0; m < DL; m++) c += wl_nz(sW[m + DL * (n + DR * (s + S * sp))]) ? 1 : 0;
        off[o + 1] = c;
    }
    __syncthreads();
    if(threadIdx.x == 0) {
        off[0] = 0;
        for(int o = 0; o < NO; o++) off[o + 1] += off[o];
    }
    __syncthreads();
    for(int o = threadIdx.x; o < NO; o += blockDim.x) {
        const int n = o / S, sp = o % S;
        int       e = off[o];
        for(int s = 0; s < S; s++)
            for(int m = 0; m < DL; m++) {
                const T w = sW[m + DL * (n + DR * (s + S * sp))];
                if(wl_nz(w)) {
                    idx[e] = (short)(m * S + s);
                    wv[e]  = w;
                    e++;
                }
            }
    }
    __syncthreads();
}

// The same list written by one thread (for a list built once and copied by every CTA of a kernel).
template<class T>
__device__ void build_wlist_serial(const T *W, int DL, int DR, int S, unsigned char *mem) {
    const int    NO  = DR * S;
    const size_t nnz = (size_t)DL * DR * S * S;
    auto         al  = [](size_t b) { return (b + 15) / 16 * 16; };
    int         *off = reinterpret_cast<int *>(mem);
    short       *idx = reinterpret_cast<short *>(mem + al(4 * (NO + 1)));
    T           *wv  = reinterpret_cast<T *>(mem + al(4 * (NO + 1)) + al(2 * nnz));
    int          e   = 0;
    for(int o = 0; o < NO; o++) {
        const int n = o / S, sp = o % S;
        off[o]      = e;
        for(int s = 0; s < S; s++)
            for(int m = 0; m < DL; m++) {
                const T w = W[m + DL * (n + DR * (s + S * sp))];
                if(wl_nz(w)) {
                    idx[e] = (short)(m * S + s);
                    wv[e]  = w;
                    e++;
                }
            }
    }
    off[NO] = e;
}
template<class T>
__global__ void wlist_global_kernel(const T *W, int DL, int DR, int S, unsigned char *out) {
    if(threadIdx.x == 0 && blockIdx.x == 0) build_wlist_serial(W, DL, DR, S, out);
}
// Views of a list block laid out as above.
template<class T>
__device__ __forceinline__ void wlist_views(unsigned char *mem, int DL, int DR, int S, int *&off, short *&idx, T *&wv) {
    const int    NO  = DR * S;
    const size_t nnz = (size_t)DL * DR * S * S;
    auto         al  = [](size_t b) { return (b + 15) / 16 * 16; };
    off              = reinterpret_cast<int *>(mem);
    idx              = reinterpret_cast<short *>(mem + al(4 * (NO + 1)));
    wv               = reinterpret_cast<T *>(mem + al(4 * (NO + 1)) + al(2 * nnz));
}

}  // namespace heff
