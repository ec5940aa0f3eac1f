// pv_output.cu — the reference's text output at GPU rates: trajectory rows
// (TrajectoryWriter::write, src/print.cpp:29-40) and the vortex block of a checkpoint
// (writeCheckpoint, src/checkpoint.cpp:86-88), byte for byte as the reference's
// `std::ostream << std::setprecision(17)` writes them.
//
// Three launches per frame:
//   1. format_rows_kernel: one thread per vortex formats its row into a fixed-stride slot
//      (pv_format.cuh: exact 17-digit %g conversion) and records its length; each block also
//      sums its rows' lengths;
//   2. scan_blocks_kernel: one block turns the block sums into exclusive block offsets and the
//      frame's total;
//   3. gather_rows_kernel: each block scans its 256 row lengths in shared memory and copies its
//      rows, which form one contiguous byte range of the frame, with consecutive threads on
//      consecutive output bytes.
// The frame then crosses to the host in one copy of exactly its size.
#include "pv_format.cuh"
#include "pv_internal.h"

namespace pvb {

namespace {

constexpr int kRowThreads = 256;

__device__ __forceinline__ int put(char *o, const char *s, int n) {
    for (int i = 0; i < n; ++i)
        o[i] = s[i];
    return n;
}

__global__ void __launch_bounds__(kRowThreads)
    format_rows_kernel(RowFormat f, char *__restrict__ staging, uint32_t *__restrict__ lengths,
                       unsigned long long *__restrict__ block_sums) {
    const size_t i = static_cast<size_t>(blockIdx.x) * kRowThreads + threadIdx.x;
    uint32_t len = 0;
    if (i < f.n) {
        char *o = staging + i * static_cast<size_t>(f.stride);
        int p = 0;
        if (f.kind == ROWS_TRAJECTORY) {
            // time,frame,index,x,y,circulation,u,v
            p += put(o, f.prefix, f.prefix_len);
            p += fmt::format_u64(i, o + p);
            o[p++] = ',';
            p += fmt::format_g17(f.x[i], o + p);
            o[p++] = ',';
            p += fmt::format_g17(f.y[i], o + p);
            o[p++] = ',';
            p += fmt::format_g17(f.g[i], o + p);
            o[p++] = ',';
            p += fmt::format_g17(f.u[i], o + p);
            o[p++] = ',';
            p += fmt::format_g17(f.v[i], o + p);
        } else {
            // x y circulation
            p += fmt::format_g17(f.x[i], o + p);
            o[p++] = ' ';
            p += fmt::format_g17(f.y[i], o + p);
            o[p++] = ' ';
            p += fmt::format_g17(f.g[i], o + p);
        }
        o[p++] = '\n';
        len = static_cast<uint32_t>(p);
        lengths[i] = len;
    }
    // block total of the row lengths
    unsigned long long s = len;
    for (int d = 16; d > 0; d >>= 1)
        s += __shfl_down_sync(0xffffffffu, s, d);
    __shared__ unsigned long long warp_sums[kRowThreads / 32];
    if ((threadIdx.x & 31) == 0)
        warp_sums[threadIdx.x >> 5] = s;
    __syncthreads();
    if (threadIdx.x == 0) {
        unsigned long long t = 0;
        for (int w = 0; w < kRowThreads / 32; ++w)
            t += warp_sums[w];
        block_sums[blockIdx.x] = t;
    }
}

// Exclusive scan of the block sums in place (one block, chunks of 1024 with a running carry);
// block_sums[blocks] receives the total.
__global__ void __launch_bounds__(1024)
    scan_blocks_kernel(unsigned long long *block_sums, size_t blocks) {
    __shared__ unsigned long long buf[1024];
    __shared__ unsigned long long carry;
    if (threadIdx.x == 0)
        carry = 0;
    __syncthreads();
    for (size_t base = 0; base < blocks; base += 1024) {
        const size_t j = base + threadIdx.x;
        const unsigned long long v = j < blocks ? block_sums[j] : 0;
        buf[threadIdx.x] = v;
        __syncthreads();
        for (int d = 1; d < 1024; d <<= 1) {  // Hillis-Steele inclusive scan
            const unsigned long long add = threadIdx.x >= d ? buf[threadIdx.x - d] : 0;
            __syncthreads();
            buf[threadIdx.x] += add;
            __syncthreads();
        }
        if (j < blocks)
            block_sums[j] = carry + buf[threadIdx.x] - v;
        __syncthreads();
        if (threadIdx.x == 1023)
            carry += buf[1023];
        __syncthreads();
    }
    if (threadIdx.x == 0)
        block_sums[blocks] = carry;
}

__global__ void __launch_bounds__(kRowThreads)
    gather_rows_kernel(const char *__restrict__ staging, const uint32_t *__restrict__ lengths,
                       const unsigned long long *__restrict__ block_offsets, size_t n,
                       int stride, char *__restrict__ out) {
    __shared__ uint32_t start[kRowThreads + 1];
    const size_t row0 = static_cast<size_t>(blockIdx.x) * kRowThreads;
    const int rows = static_cast<int>(min(static_cast<size_t>(kRowThreads), n - row0));
    const uint32_t len = threadIdx.x < rows ? lengths[row0 + threadIdx.x] : 0;
    start[threadIdx.x + 1] = len;
    if (threadIdx.x == 0)
        start[0] = 0;
    __syncthreads();
    for (int d = 1; d < kRowThreads; d <<= 1) {  // inclusive scan of start[1..256]
        const uint32_t add = threadIdx.x >= d ? start[threadIdx.x + 1 - d] : 0;
        __syncthreads();
        start[threadIdx.x + 1] += add;
        __syncthreads();
    }
    const uint32_t total = start[rows];
    char *dst = out + block_offsets[blockIdx.x];
    for (uint32_t b = threadIdx.x; b < total; b += kRowThreads) {
        int lo = 0, hi = rows - 1;  // the row r with start[r] <= b < start[r + 1]
        while (lo < hi) {
            const int mid = (lo + hi + 1) >> 1;
            if (start[mid] <= b)
                lo = mid;
            else
                hi = mid - 1;
        }
        dst[b] = staging[(row0 + lo) * static_cast<size_t>(stride) + (b - start[lo])];
    }
}

}  // namespace

int format_prefix(double time, uint64_t frame, char *out) {
    int p = fmt::format_g17(time, out);
    out[p++] = ',';
    p += fmt::format_u64(frame, out + p);
    out[p++] = ',';
    return p;
}

cudaError_t launch_format_rows(const RowFormat &f, char *staging, uint32_t *lengths,
                               unsigned long long *block_sums, char *out, cudaStream_t stream) {
    const size_t blocks = (f.n + kRowThreads - 1) / kRowThreads;
    if (blocks == 0) {
        return cudaMemsetAsync(block_sums, 0, sizeof(unsigned long long), stream);
    }
    format_rows_kernel<<<static_cast<unsigned>(blocks), kRowThreads, 0, stream>>>(
        f, staging, lengths, block_sums);
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess)
        return e;
    scan_blocks_kernel<<<1, 1024, 0, stream>>>(block_sums, blocks);
    if ((e = cudaGetLastError()) != cudaSuccess)
        return e;
    gather_rows_kernel<<<static_cast<unsigned>(blocks), kRowThreads, 0, stream>>>(
        staging, lengths, block_sums, f.n, f.stride, out);
    return cudaGetLastError();
}

}  // namespace pvb
