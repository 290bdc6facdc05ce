// Exceptions of rec buffers (src/cor/eng/hzl_de_cmp.cpp:28-77): after the FFOR blocks of a rec buffer are
// unpacked in place of their 1024 values, each block's exceptions overwrite the values at their positions.
#include "fls_rec.h"
#include "fls_runtime.h"

namespace flsgpu {

// One warp per block: exc_c u16 positions at src + exc_off, then exc_c values of `eb` bytes; both may sit at any
// byte address inside the page.
__global__ void k_rec_patch(const uint8_t* __restrict__ src, const RecBlock* __restrict__ blocks, uint32_t n_blocks,
                            uint32_t eb, uint8_t* __restrict__ dst) {
	const uint32_t lane = threadIdx.x & 31u;
	for (uint32_t b = blockIdx.x * (blockDim.x / 32) + (threadIdx.x >> 5); b < n_blocks; b += gridDim.x * (blockDim.x / 32)) {
		const RecBlock  k    = blocks[b];
		const uint8_t*  pos  = src + k.exc_off;
		const uint8_t*  vals = pos + 2ull * k.exc_c;
		uint8_t*        out  = dst + static_cast<uint64_t>(b) * 1024 * eb;
		for (uint32_t i = lane; i < k.exc_c; i += 32) {
			const uint32_t p = static_cast<uint32_t>(pos[2 * i]) | (static_cast<uint32_t>(pos[2 * i + 1]) << 8);
			if (p >= 1024) { continue; }
			for (uint32_t j = 0; j < eb; ++j) { out[p * eb + j] = vals[static_cast<uint64_t>(i) * eb + j]; }
		}
	}
}

cudaError_t launch_rec_patch(const uint8_t* src, const RecBlock* blocks, uint32_t n_blocks, uint32_t eb, uint8_t* dst,
                             cudaStream_t s) {
	if (n_blocks == 0) { return cudaSuccess; }
	const unsigned grid = (n_blocks + 7) / 8 < 1024u ? (n_blocks + 7) / 8 : 1024u;
	k_rec_patch<<<grid, 256, 0, s>>>(src, blocks, n_blocks, eb, dst);
	++launch_counter();
	return cudaGetLastError();
}

} // namespace flsgpu
