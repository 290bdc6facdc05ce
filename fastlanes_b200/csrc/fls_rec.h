// Rec buffers (the reference's page-level "record" compression, src/cor/eng/hzl_cmp.cpp:43-127 writes them,
// src/cor/eng/hzl_de_cmp.cpp:28-77 reads them): a chain of blocks, each a 12-byte rec_hdr {bw u8, pad u8, exc_c
// u16, base[8]} (include/fls/cor/lyt/rec_hdr.hpp:7-13) followed by
//   * bw = 255: base holds a byte count; that many raw bytes follow and end the chain;
//   * any other bw: 1024 values of the buffer's element type FFOR-packed at that bit width (bw * 128 bytes,
//     generated ffor, positions kept), then exc_c u16 positions and exc_c values that replace the unpacked ones.
// The element type is uint64 for 64-bit values and dictionary entries, idx_t = uint32 for run codes
// (include/fls/common/alias.hpp:17) and uint16 for the rsum bases of RLE REC2 pages.
#pragma once

#include <cstdint>
#include <cuda_runtime.h>
#include <vector>

namespace flsgpu {

struct RecBlock {
	uint64_t exc_off; // byte offset of the block's exception positions inside the rec buffer
	uint32_t exc_c;
	uint32_t pad;
};

cudaError_t launch_rec_patch(const uint8_t* src, const RecBlock* blocks, uint32_t n_blocks, uint32_t eb, uint8_t* dst,
                             cudaStream_t s);

// Decode the rec buffer at d_src (device, `size` bytes; h_src: the same bytes on the host, for walking the chain)
// with element size eb (2, 4 or 8) into a new device buffer (*d_out, cudaMallocAsync on s, to be freed by the
// caller) of *out_size decoded bytes.  The FFOR blocks run through the engine's own unffor kernels.
int rec_decode(const uint8_t* d_src, const uint8_t* h_src, uint64_t size, uint32_t eb, uint8_t** d_out,
               uint64_t* out_size, cudaStream_t s);

// True when the rec buffer is a single raw block (nothing to decode): *raw_off / *raw_size locate its bytes.
bool rec_is_raw(const uint8_t* h_src, uint64_t size, uint64_t* raw_off, uint64_t* raw_size);

} // namespace flsgpu
