// Selections of filter plans (predicate pushdown): bitmaps -> index lists, bitmap combination, and the
// intersection of index lists (src/primitive/predicate/equal.cpp:12-28 and :100-119 of the reference).  One
// warp per vector; a vector's bitmap is 32 u32 words, one per lane.
#include "fls_b200.h"
#include "fls_plan.h"
#include "fls_runtime.h"
#include "fls_strings.cuh"

namespace flsgpu {

namespace {

// Positions of the set bits of the vector's bitmap (lane l holds word l, bits 32l .. 32l + 31) in ascending
// order into idx; returns the count (every lane).
__device__ __forceinline__ uint32_t compact_bits(uint32_t word, uint32_t lane, uint16_t* idx) {
	const uint32_t c   = __popc(word);
	const uint32_t inc = warp_inclusive_scan(c, lane);
	uint32_t       o   = inc - c;
	while (word) {
		const uint32_t b = __ffs(word) - 1;
		idx[o++]         = static_cast<uint16_t>(32 * lane + b);
		word &= word - 1;
	}
	return __shfl_sync(0xFFFFFFFFu, inc, 31);
}

__global__ void k_bitmap_to_selection(const uint32_t* __restrict__ bm, uint64_t n_vec, uint16_t* __restrict__ idx,
                                      uint16_t* __restrict__ count) {
	const uint32_t lane = threadIdx.x & 31u;
	const uint64_t nw   = static_cast<uint64_t>(gridDim.x) * (blockDim.x / 32);
	for (uint64_t v = static_cast<uint64_t>(blockIdx.x) * (blockDim.x / 32) + threadIdx.x / 32; v < n_vec; v += nw) {
		const uint32_t n = compact_bits(bm[32 * v + lane], lane, idx + 1024 * v);
		if (lane == 0) { count[v] = static_cast<uint16_t>(n); }
	}
}

__global__ void k_bitmap_combine(const uint32_t* __restrict__ a, const uint32_t* __restrict__ b, uint32_t* out,
                                 uint64_t n_words, int op) {
	for (uint64_t i = static_cast<uint64_t>(blockIdx.x) * blockDim.x + threadIdx.x; i < n_words;
	     i += static_cast<uint64_t>(gridDim.x) * blockDim.x) {
		const uint32_t x = a[i], y = b[i];
		out[i]           = op == FLS_BITMAP_AND ? (x & y) : op == FLS_BITMAP_OR ? (x | y) : (x & ~y);
	}
}

// Bits of an index list in shared memory (32 words per warp); false when a position or the count is out of
// range.
__device__ __forceinline__ bool list_bits(const uint16_t* idx, uint32_t n, uint32_t* bits, uint32_t lane) {
	bits[lane] = 0;
	__syncwarp();
	bool bad = n > 1024;
	n        = n > 1024 ? 1024 : n;
	for (uint32_t i = lane; i < n; i += 32) {
		const uint32_t p = idx[i];
		if (p < 1024) {
			atomicOr(bits + p / 32, 1u << (p % 32));
		} else {
			bad = true;
		}
	}
	__syncwarp();
	return !__any_sync(0xFFFFFFFFu, bad);
}

__global__ void k_selection_and(const uint16_t* __restrict__ i0, const uint16_t* __restrict__ c0,
                                const uint16_t* __restrict__ i1, const uint16_t* __restrict__ c1, uint16_t* io,
                                uint16_t* co, uint64_t n_vec, int* status) {
	__shared__ uint32_t bits[8][2][32];
	const uint32_t      lane = threadIdx.x & 31u, warp = threadIdx.x / 32;
	const uint64_t      nw   = static_cast<uint64_t>(gridDim.x) * (blockDim.x / 32);
	for (uint64_t v = static_cast<uint64_t>(blockIdx.x) * (blockDim.x / 32) + warp; v < n_vec; v += nw) {
		const bool ok0 = list_bits(i0 + 1024 * v, c0[v], bits[warp][0], lane);
		const bool ok1 = list_bits(i1 + 1024 * v, c1[v], bits[warp][1], lane);
		if (!(ok0 && ok1) && lane == 0) { atomicOr(status, STATUS_BAD_INDEX); }
		const uint32_t n = compact_bits(bits[warp][0][lane] & bits[warp][1][lane], lane, io + 1024 * v);
		if (lane == 0) { co[v] = static_cast<uint16_t>(n); }
		__syncwarp();
	}
}

unsigned grid_for(uint64_t warps_needed) {
	const Device* d    = current_device();
	const uint64_t cap = static_cast<uint64_t>(d ? d->sm_count : 148) * 8; // 8 CTAs of 8 warps per SM
	const uint64_t g   = (warps_needed + 7) / 8;
	return static_cast<unsigned>(g < cap ? (g ? g : 1) : cap);
}

} // namespace

} // namespace flsgpu

extern "C" {

int fls_gpu_bitmap_to_selection(const uint64_t* d_bitmaps, uint64_t n_vec, uint16_t* d_idx, uint16_t* d_count,
                                fls_stream_t stream) {
	using namespace flsgpu;
	if (n_vec == 0) { return FLS_OK; }
	if (!d_bitmaps || !d_idx || !d_count) { return FLS_ERR_ARG; }
	k_bitmap_to_selection<<<grid_for(n_vec), 256, 0, static_cast<cudaStream_t>(stream)>>>(
	    reinterpret_cast<const uint32_t*>(d_bitmaps), n_vec, d_idx, d_count);
	++launch_counter();
	return cudaGetLastError() == cudaSuccess ? FLS_OK : FLS_ERR_CUDA;
}

int fls_gpu_bitmap_combine(const uint64_t* d_a, const uint64_t* d_b, uint64_t* d_out, uint64_t n_vec, int op,
                           fls_stream_t stream) {
	using namespace flsgpu;
	if (op < FLS_BITMAP_AND || op > FLS_BITMAP_ANDNOT) { return FLS_ERR_ARG; }
	if (n_vec == 0) { return FLS_OK; }
	if (!d_a || !d_b || !d_out) { return FLS_ERR_ARG; }
	const uint64_t words = 32 * n_vec;
	k_bitmap_combine<<<grid_for(words / 32), 256, 0, static_cast<cudaStream_t>(stream)>>>(
	    reinterpret_cast<const uint32_t*>(d_a), reinterpret_cast<const uint32_t*>(d_b),
	    reinterpret_cast<uint32_t*>(d_out), words, op);
	++launch_counter();
	return cudaGetLastError() == cudaSuccess ? FLS_OK : FLS_ERR_CUDA;
}

int fls_gpu_selection_and(const uint16_t* d_idx0, const uint16_t* d_count0, const uint16_t* d_idx1,
                          const uint16_t* d_count1, uint16_t* d_idx_out, uint16_t* d_count_out, uint64_t n_vec,
                          fls_stream_t stream) {
	using namespace flsgpu;
	if (n_vec == 0) { return FLS_OK; }
	if (!d_idx0 || !d_count0 || !d_idx1 || !d_count1 || !d_idx_out || !d_count_out) { return FLS_ERR_ARG; }
	Device* d = current_device();
	if (!d) { return FLS_ERR_CUDA; }
	k_selection_and<<<grid_for(n_vec), 256, 0, static_cast<cudaStream_t>(stream)>>>(
	    d_idx0, d_count0, d_idx1, d_count1, d_idx_out, d_count_out, n_vec, d->status);
	++launch_counter();
	return cudaGetLastError() == cudaSuccess ? FLS_OK : FLS_ERR_CUDA;
}

} // extern "C"
