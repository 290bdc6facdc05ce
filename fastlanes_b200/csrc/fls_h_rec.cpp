// Host side of rec buffer decoding (format in fls_rec.h): walk the block chain, unpack every FFOR block with the
// engine's unffor kernels (one batched launch), patch the exceptions, copy the raw tail.
#include "fls_rec.h"
#include "fls_b200.h"

#include <cstring>

namespace flsgpu {

namespace {

struct Walk {
	std::vector<uint64_t> packed_off; // per FFOR block, byte offset of its packed words
	std::vector<uint8_t>  bw;
	std::vector<uint8_t>  base;       // eb bytes per block
	std::vector<RecBlock> exc;
	uint64_t              tail_off = 0, tail_size = 0;
};

int walk(const uint8_t* h, uint64_t size, uint32_t eb, Walk* w) {
	uint64_t pos = 0;
	while (true) {
		if (pos + 12 > size) { return FLS_ERR_FORMAT; }
		const uint8_t bw    = h[pos];
		uint16_t      exc_c = 0;
		std::memcpy(&exc_c, h + pos + 2, 2);
		const uint8_t* base = h + pos + 4;
		pos += 12;
		if (bw == 255) {
			uint64_t sz = 0;
			std::memcpy(&sz, base, 8);
			if (sz > size - pos) { return FLS_ERR_FORMAT; }
			w->tail_off  = pos;
			w->tail_size = sz;
			return FLS_OK;
		}
		if (bw > 8 * eb || exc_c > 1024) { return FLS_ERR_FORMAT; }
		const uint64_t packed = 128ull * bw;
		const uint64_t excb   = static_cast<uint64_t>(exc_c) * (2 + eb);
		if (packed + excb > size - pos) { return FLS_ERR_FORMAT; }
		w->packed_off.push_back(pos);
		w->bw.push_back(bw);
		w->base.insert(w->base.end(), base, base + eb);
		w->exc.push_back(RecBlock {pos + packed, exc_c, 0});
		pos += packed + excb;
	}
}

} // namespace

bool rec_is_raw(const uint8_t* h, uint64_t size, uint64_t* raw_off, uint64_t* raw_size) {
	if (size < 12 || h[0] != 255) { return false; }
	uint64_t sz = 0;
	std::memcpy(&sz, h + 4, 8);
	if (sz > size - 12) { return false; }
	*raw_off  = 12;
	*raw_size = sz;
	return true;
}

int rec_decode(const uint8_t* d_src, const uint8_t* h_src, uint64_t size, uint32_t eb, uint8_t** d_out,
               uint64_t* out_size, cudaStream_t s) {
	if ((eb != 2 && eb != 4 && eb != 8) || !d_out || !out_size) { return FLS_ERR_ARG; }
	Walk w;
	int  rc = walk(h_src, size, eb, &w);
	if (rc != FLS_OK) { return rc; }
	const uint64_t nb   = w.bw.size();
	const uint64_t full = nb * 1024ull * eb;
	*out_size           = full + w.tail_size;
	*d_out              = nullptr;
	if (cudaMallocAsync(reinterpret_cast<void**>(d_out), *out_size + 16, s) != cudaSuccess) { return FLS_ERR_CUDA; }
	if (nb > 0) {
		// the unffor entry point wants its packed base 4-byte aligned: offsets are taken from the aligned-down
		// start of the rec buffer
		const uint8_t* base_ptr = reinterpret_cast<const uint8_t*>(reinterpret_cast<uintptr_t>(d_src) & ~uintptr_t(15));
		const uint64_t shift    = static_cast<uint64_t>(d_src - base_ptr);
		std::vector<uint64_t> off(nb);
		for (uint64_t i = 0; i < nb; ++i) { off[i] = w.packed_off[i] + shift; }
		const size_t bytes = nb * 8 + nb + nb * eb + nb * sizeof(RecBlock);
		uint8_t*     tmp   = nullptr;
		if (cudaMallocAsync(reinterpret_cast<void**>(&tmp), bytes + 64, s) != cudaSuccess) { return FLS_ERR_CUDA; }
		uint64_t* d_off  = reinterpret_cast<uint64_t*>(tmp);
		RecBlock* d_exc  = reinterpret_cast<RecBlock*>(tmp + nb * 8);
		uint8_t*  d_base = tmp + nb * 8 + nb * sizeof(RecBlock);
		uint8_t*  d_bw   = d_base + nb * eb;
		// copies from pageable host memory are staged before cudaMemcpyAsync returns
		bool ok = cudaMemcpyAsync(d_off, off.data(), nb * 8, cudaMemcpyHostToDevice, s) == cudaSuccess &&
		          cudaMemcpyAsync(d_exc, w.exc.data(), nb * sizeof(RecBlock), cudaMemcpyHostToDevice, s) == cudaSuccess &&
		          cudaMemcpyAsync(d_base, w.base.data(), nb * eb, cudaMemcpyHostToDevice, s) == cudaSuccess &&
		          cudaMemcpyAsync(d_bw, w.bw.data(), nb, cudaMemcpyHostToDevice, s) == cudaSuccess;
		if (ok) {
			rc = eb == 8 ? fls_gpu_unffor_u64(reinterpret_cast<const uint64_t*>(base_ptr), reinterpret_cast<uint64_t*>(*d_out),
			                                  d_bw, reinterpret_cast<const uint64_t*>(d_base), d_off, nb, FLS_TRANSPOSED, s)
			     : eb == 4 ? fls_gpu_unffor_u32(reinterpret_cast<const uint32_t*>(base_ptr), reinterpret_cast<uint32_t*>(*d_out),
			                                  d_bw, reinterpret_cast<const uint32_t*>(d_base), d_off, nb, FLS_TRANSPOSED, s)
			               : fls_gpu_unffor_u16(reinterpret_cast<const uint16_t*>(base_ptr), reinterpret_cast<uint16_t*>(*d_out),
			                                  d_bw, reinterpret_cast<const uint16_t*>(d_base), d_off, nb, FLS_TRANSPOSED, s);
			ok = rc == FLS_OK && launch_rec_patch(d_src, d_exc, static_cast<uint32_t>(nb), eb, *d_out, s) == cudaSuccess;
		}
		cudaFreeAsync(tmp, s);
		if (!ok) { return rc != FLS_OK ? rc : FLS_ERR_CUDA; }
	}
	if (w.tail_size > 0 &&
	    cudaMemcpyAsync(*d_out + full, d_src + w.tail_off, w.tail_size, cudaMemcpyDeviceToDevice, s) != cudaSuccess) {
		return FLS_ERR_CUDA;
	}
	return FLS_OK;
}

} // namespace flsgpu
