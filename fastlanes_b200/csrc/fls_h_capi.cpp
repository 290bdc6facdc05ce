// The reference's C API (include/fastlanes.h) served by the GPU engine, with host buffers on both sides.
//
// encode_from_memory follows the single-column encoder of the reference (src/connection.cpp:150-167,
// src/encoder/single_col_encoder.cpp:9-34, src/encoder/exp_col_encoder.cpp:40-64): the page of the chosen
// expression, built from whole 1024-value vectors; the per-vector steps run on the GPU
//   UNCOMPRESSED (id 0): transpose_i                         -> [values]
//   FFOR        (id 1): transpose_i, analyze, ffor           -> [bw][base][packed]
//   DELTA       (id 11): transpose_i, lane bases = row 0, unrsum, analyze, ffor
//                                                            -> [lane bases][bw][base][packed]
// (RPN tables include/fls/cor/exp/ffor/ffor_exp.hpp:35-53, include/fls/cor/exp/delta/delta_exp.hpp:39-56;
// primitives src/cor/prm/{trs,rsum,ffor}/*_compress.cpp, src/cor/prm/ffor/ffor_analyze.cpp:77-102) and the
// host writes the page framing (src/cor/eng/compressor.cpp:68-86).
// decode_to_memory places the page in device memory with its packed buffer on a 16-byte boundary, decodes it
// with the page engine and copies the values back.
#include "fastlanes.h"
#include "fls_b200.h"
#include "fls_page.h"
#include "fls_rec.h"
#include "fls_runtime.h"

#include <algorithm>
#include <cstring>
#include <cuda_runtime.h>
#include <mutex>
#include <vector>

struct Connection {
	int magic = 0x464C5342; // "FLSB"
};

namespace flsgpu {
namespace {

cudaStream_t api_stream() {
	static cudaStream_t s[64] {};
	static std::mutex   mu;
	int                 d = 0;
	if (cudaGetDevice(&d) != cudaSuccess || d < 0 || d >= 64) { return nullptr; }
	std::lock_guard<std::mutex> lk(mu);
	if (!s[d]) { cudaStreamCreateWithFlags(&s[d], cudaStreamNonBlocking); }
	return s[d];
}

struct DevBuf {
	void*        p = nullptr;
	cudaStream_t s = nullptr;
	explicit DevBuf(cudaStream_t st) : s(st) {}
	bool alloc(size_t n) { return cudaMallocAsync(&p, n ? n : 16, s) == cudaSuccess; }
	~DevBuf() {
		if (p) { cudaFreeAsync(p, s); }
	}
	template <class T>
	T* as() const {
		return static_cast<T*>(p);
	}
};

// Size of a page from its bytes: the last buffer is always the stream's packed (or raw) buffer, so its size is
// the last vector's entry point plus that vector's packed size.
int page_size_of(const uint8_t* page, PageInfo* pi, uint64_t* size, int value_width) {
	int rc = parse_page_header(page, 8 + 4 * 6, pi);
	if (rc != FLS_OK) { return rc; }
	const ExprLayout* L    = pi->layout;
	const uint32_t    last = pi->arr_c - 1;
	if (pi->vec_c == 0) {
		*size = pi->off[last];
		return FLS_OK;
	}
	const uint32_t v  = pi->vec_c - 1u;
	auto           ep = [&](uint32_t vv, uint32_t i) -> uint64_t {
        if (vv == 0) { return 0; }
        uint32_t x;
        std::memcpy(&x, page + pi->ep_off + 4ull * ((vv - 1) * pi->arr_c + i), 4);
        return x;
	};
	const uint32_t ws = L->ws ? L->ws : static_cast<uint32_t>(value_width);
	uint64_t       part;
	if (L->enc == ENC_RAW) {
		part = ws * 128ull;
	} else {
		part = page[pi->off[L->ib_bw] + ep(v, L->ib_bw)] * 128ull;
	}
	*size = pi->off[last] + ep(v, last) + part;
	return FLS_OK;
}

template <class T>
int encode_t(const T* in, uint64_t n, uint64_t cap, uint8_t* out, uint64_t* out_size, uint64_t* mtd_size, bool sgn,
             uint8_t expr) {
	constexpr int      W     = sizeof(T) * 8;
	constexpr uint32_t L     = 1024 / W;
	const uint64_t     n_vec = n / 1024;
	if (n_vec > 0xFFFFu) { return FLS_ERR_ARG; }
	uint8_t  exp_t, arr_c;
	switch (expr) {
	case 0: exp_t = 2, arr_c = 1; break;
	case 1: exp_t = 4, arr_c = 3; break;
	case 11: exp_t = 5, arr_c = 4; break;
	default: return FLS_ERR_UNSUPPORTED;
	}
	cudaStream_t s = api_stream();
	if (!s) { return FLS_ERR_CUDA; }
	const uint64_t bytes = n_vec * 1024 * sizeof(T);
	DevBuf         d_in(s), d_tr(s), d_delta(s), d_bw(s), d_base(s), d_off(s), d_packed(s);
	std::vector<uint8_t>  bw(n_vec);
	std::vector<T>        base(n_vec);
	std::vector<uint64_t> off(n_vec);
	std::vector<T>        lane_bases;
	uint64_t              packed_total = 0;
	if (n_vec > 0) {
		if (!d_in.alloc(bytes) || !d_tr.alloc(bytes)) { return FLS_ERR_CUDA; }
		cudaMemcpyAsync(d_in.p, in, bytes, cudaMemcpyHostToDevice, s);
		int rc;
		if constexpr (W == 64) {
			rc = fls_gpu_transpose_i_u64(d_in.as<uint64_t>(), d_tr.as<uint64_t>(), n_vec, s);
		} else {
			rc = fls_gpu_transpose_i_u32(d_in.as<uint32_t>(), d_tr.as<uint32_t>(), n_vec, s);
		}
		if (rc != FLS_OK) { return rc; }
		if (expr != 0) {
			const T* src = d_tr.as<T>();
			if (expr == 11) {
				lane_bases.resize(n_vec * L);
				cudaMemcpy2DAsync(lane_bases.data(), 128, d_tr.p, 1024 * sizeof(T), 128, n_vec, cudaMemcpyDeviceToHost,
				                  s);
				if (!d_delta.alloc(bytes)) { return FLS_ERR_CUDA; }
				if constexpr (W == 64) {
					rc = fls_gpu_unrsum_u64(d_tr.as<uint64_t>(), d_delta.as<uint64_t>(), n_vec, s);
				} else {
					rc = fls_gpu_unrsum_u32(d_tr.as<uint32_t>(), d_delta.as<uint32_t>(), n_vec, s);
				}
				if (rc != FLS_OK) { return rc; }
				src = d_delta.as<T>();
			}
			if (!d_bw.alloc(n_vec) || !d_base.alloc(n_vec * sizeof(T)) || !d_off.alloc(n_vec * 8)) {
				return FLS_ERR_CUDA;
			}
			if constexpr (W == 64) {
				rc = fls_gpu_analyze_u64(reinterpret_cast<const uint64_t*>(src), d_bw.as<uint8_t>(),
				                         d_base.as<uint64_t>(), n_vec, sgn, s);
			} else {
				rc = fls_gpu_analyze_u32(reinterpret_cast<const uint32_t*>(src), d_bw.as<uint8_t>(),
				                         d_base.as<uint32_t>(), n_vec, sgn, s);
			}
			if (rc != FLS_OK) { return rc; }
			cudaMemcpyAsync(bw.data(), d_bw.p, n_vec, cudaMemcpyDeviceToHost, s);
			cudaMemcpyAsync(base.data(), d_base.p, n_vec * sizeof(T), cudaMemcpyDeviceToHost, s);
			if (cudaStreamSynchronize(s) != cudaSuccess) { return FLS_ERR_CUDA; }
			for (uint64_t v = 0; v < n_vec; ++v) {
				off[v] = packed_total;
				packed_total += bw[v] * 128ull;
			}
			if (!d_packed.alloc(packed_total + 16)) { return FLS_ERR_CUDA; }
			cudaMemcpyAsync(d_off.p, off.data(), n_vec * 8, cudaMemcpyHostToDevice, s);
			if constexpr (W == 64) {
				rc = fls_gpu_ffor_u64(reinterpret_cast<const uint64_t*>(src), d_packed.as<uint64_t>(), d_bw.as<uint8_t>(),
				                      d_base.as<uint64_t>(), d_off.as<uint64_t>(), n_vec, s);
			} else {
				rc = fls_gpu_ffor_u32(reinterpret_cast<const uint32_t*>(src), d_packed.as<uint32_t>(), d_bw.as<uint8_t>(),
				                      d_base.as<uint32_t>(), d_off.as<uint64_t>(), n_vec, s);
			}
			if (rc != FLS_OK) { return rc; }
		}
	}
	// page framing: header, buffer offsets, entry points of vectors 1.., buffers
	std::vector<uint64_t> buf_len(arr_c);
	if (expr == 0) {
		buf_len[0] = bytes;
	} else {
		const uint32_t first = expr == 11 ? 1 : 0;
		if (expr == 11) { buf_len[0] = n_vec * 128; }
		buf_len[first]     = n_vec;
		buf_len[first + 1] = n_vec * sizeof(T);
		buf_len[first + 2] = packed_total;
	}
	const uint64_t meta = 8 + 4ull * arr_c + 4ull * arr_c * (n_vec ? n_vec - 1 : 0);
	uint64_t       total = meta;
	for (auto b : buf_len) { total += b; }
	if (out_size) { *out_size = total; }
	if (mtd_size) { *mtd_size = meta; }
	if (total > cap || !out) {
		cudaStreamSynchronize(s);
		return FLS_ERR_ARG;
	}
	uint8_t* p = out;
	std::memset(p, 0, 8);
	p[0]                 = exp_t;
	p[1]                 = 1; // NO_PATCH / UNCOMPRESSED variant
	const uint16_t vec_c = static_cast<uint16_t>(n_vec);
	std::memcpy(p + 4, &vec_c, 2);
	uint64_t boff[4];
	boff[0] = meta;
	for (uint32_t i = 1; i < arr_c; ++i) { boff[i] = boff[i - 1] + buf_len[i - 1]; }
	for (uint32_t i = 0; i < arr_c; ++i) {
		const uint32_t o = static_cast<uint32_t>(boff[i]);
		std::memcpy(p + 8 + 4 * i, &o, 4);
	}
	uint8_t* ep = p + 8 + 4 * arr_c;
	for (uint64_t v = 1; v < n_vec; ++v) {
		uint32_t e[4];
		if (expr == 0) {
			e[0] = static_cast<uint32_t>(v * 1024 * sizeof(T));
		} else {
			uint32_t j = 0;
			if (expr == 11) { e[j++] = static_cast<uint32_t>(v * 128); }
			e[j++] = static_cast<uint32_t>(v);
			e[j++] = static_cast<uint32_t>(v * sizeof(T));
			e[j++] = static_cast<uint32_t>(off[v]);
		}
		std::memcpy(ep + 4ull * arr_c * (v - 1), e, 4ull * arr_c);
	}
	if (n_vec > 0) {
		if (expr == 0) {
			cudaMemcpyAsync(p + boff[0], d_tr.p, bytes, cudaMemcpyDeviceToHost, s);
		} else {
			const uint32_t first = expr == 11 ? 1 : 0;
			if (expr == 11) { std::memcpy(p + boff[0], lane_bases.data(), n_vec * 128); }
			std::memcpy(p + boff[first], bw.data(), n_vec);
			std::memcpy(p + boff[first + 1], base.data(), n_vec * sizeof(T));
			cudaMemcpyAsync(p + boff[first + 2], d_packed.p, packed_total, cudaMemcpyDeviceToHost, s);
		}
	}
	return cudaStreamSynchronize(s) == cudaSuccess ? FLS_OK : FLS_ERR_CUDA;
}

// The three streams of the host decode pipeline of the current device: copies in, decode, copies out.
constexpr uint32_t kPipeEvents = 256;    // three per chunk: enough for a 65,535-vector page of 8-byte values
// A chunk's copy in waits for the copy out of the chunk kPipeLead places before it.  Copies in are half the
// bytes of copies out: issued all at once they take half the link for the first part of the call and the
// copies out then run alone; paced, both directions stay busy for the whole call.
constexpr uint32_t kPipeLead = 2;
constexpr uint32_t kPipeIds     = 65536; // the identity work queue of a page's vectors, uploaded once
struct HostPipe {
	cudaStream_t in = nullptr, dec = nullptr, out = nullptr;
	cudaEvent_t  ev[kPipeEvents] {};
	uint32_t*    ids = nullptr; // device: ids[v] = v
	std::mutex   call;          // one host-page decode at a time per device (the events are shared)
};
HostPipe* host_pipe() {
	static HostPipe   p[64];
	static std::mutex mu;
	int               d = 0;
	if (cudaGetDevice(&d) != cudaSuccess || d < 0 || d >= 64) { return nullptr; }
	std::lock_guard<std::mutex> lk(mu);
	HostPipe&                   h = p[d];
	if (!h.in) {
		if (cudaStreamCreateWithFlags(&h.in, cudaStreamNonBlocking) != cudaSuccess ||
		    cudaStreamCreateWithFlags(&h.dec, cudaStreamNonBlocking) != cudaSuccess ||
		    cudaStreamCreateWithFlags(&h.out, cudaStreamNonBlocking) != cudaSuccess) {
			h.in = nullptr;
			return nullptr;
		}
		for (auto& e : h.ev) {
			if (cudaEventCreateWithFlags(&e, cudaEventDisableTiming) != cudaSuccess) {
				h.in = nullptr;
				return nullptr;
			}
		}
		std::vector<uint32_t> ids(kPipeIds);
		for (uint32_t v = 0; v < kPipeIds; ++v) { ids[v] = v; }
		if (cudaMalloc(&h.ids, 4ull * kPipeIds) != cudaSuccess ||
		    cudaMemcpy(h.ids, ids.data(), 4ull * kPipeIds, cudaMemcpyHostToDevice) != cudaSuccess) {
			h.in = nullptr;
			return nullptr;
		}
		// this process's stream-ordered allocations keep their memory between calls instead of returning it
		// at every synchronisation (a call maps its staging buffers once, not on every page)
		cudaMemPool_t pool = nullptr;
		uint64_t      keep = ~0ull;
		if (cudaDeviceGetDefaultMemPool(&pool, d) == cudaSuccess) {
			cudaMemPoolSetAttribute(pool, cudaMemPoolAttrReleaseThreshold, &keep);
		}
	}
	return &h;
}

// Decode a page held in host memory into host memory.  The header is parsed from the host copy and the page's
// small per-vector buffers go over whole; the vectors then go through in chunks of output growing from about
// 1 MB to about 16 MB: each chunk's slice of the largest buffer is copied in on one stream, decoded on a second
// (a queue of the chunk's vector ids) and copied out on a third, so the copies in both directions and the
// kernels overlap (with pinned host buffers).
int decode_host_page(const uint8_t* page, uint64_t page_size, void* out, uint64_t out_cap, uint8_t dt,
                     uint64_t* n_values) {
	const int w = value_width_of(dt);
	if (!page || w == 0) { return FLS_ERR_UNSUPPORTED; }
	PageInfo pi;
	uint64_t computed = 0;
	int      rc       = page_size_of(page, &pi, &computed, w);
	if (rc != FLS_OK) { return rc; }
	// doubles: their 64-bit patterns, through every layout but RLE's rec-compressed run values (the reference
	// has no rec buffers of doubles) and ALP (no layout here: the ALP library is not part of the reference snapshot)
	if (dt == DOUBLE && pi.layout->ib_rec != kNoBuf && pi.layout->post == POST_RLE) { return FLS_ERR_UNSUPPORTED; }
	if (page_size == 0) { page_size = computed; }
	if (computed > page_size) { return FLS_ERR_FORMAT; }
	rc = finish_page_info(&pi, page_size);
	if (rc != FLS_OK) { return rc; }
	// the C API carries no dictionary
	if (pi.layout->post == POST_DICT || pi.layout->post == POST_RLE_DICT) { return FLS_ERR_FORMAT; }
	const uint64_t sz        = static_cast<uint64_t>(w / 8);
	const uint64_t out_bytes = static_cast<uint64_t>(pi.vec_c) * 1024 * sz;
	if (n_values) { *n_values = static_cast<uint64_t>(pi.vec_c) * 1024; }
	if (out_cap < out_bytes || !out) { return FLS_ERR_ARG; }
	if (pi.vec_c == 0) { return FLS_OK; }
	HostPipe* hp = host_pipe();
	if (!hp) { return FLS_ERR_CUDA; }
	std::lock_guard<std::mutex> call_lock(hp->call);
	const uint32_t shift = static_cast<uint32_t>((16 - pi.off[pi.layout->ib_packed] % 16) % 16);
	DevBuf         d_page(hp->in), d_out(hp->in);
	if (!d_page.alloc(page_size + 32) || !d_out.alloc(out_bytes)) { return FLS_ERR_CUDA; }
	uint8_t* dp = d_page.as<uint8_t>() + shift;
	// _REC variants: the rec-compressed value buffer goes over whole and is decoded first (on the copy stream,
	// so every chunk's decode is ordered after it)
	const int rec_b = pi.layout->ib_rec != kNoBuf ? pi.layout->ib_rec : -1;
	DevBuf    d_rec(hp->in);
	uint64_t  rec_n = 0;
	if (rec_b >= 0) {
		if (cudaMemcpyAsync(dp + pi.off[rec_b], page + pi.off[rec_b], pi.size[rec_b], cudaMemcpyHostToDevice, hp->in) !=
		    cudaSuccess) {
			return FLS_ERR_CUDA;
		}
		uint8_t*       rb = nullptr;
		const uint32_t eb = pi.layout->post == POST_RLE_DICT ? 4u : static_cast<uint32_t>(w / 8);
		rc                = rec_decode(dp + pi.off[rec_b], page + pi.off[rec_b], pi.size[rec_b], eb, &rb, &rec_n, hp->in);
		d_rec.p           = rb;
		if (rc != FLS_OK) { return rc; }
	}
	// REC2: the u16 rsum bases are a second rec buffer
	const int rec2_b = pi.layout->ib_rec2 != kNoBuf ? pi.layout->ib_rec2 : -1;
	DevBuf    d_rec2(hp->in);
	uint64_t  rec2_n = 0;
	if (rec2_b >= 0) {
		if (cudaMemcpyAsync(dp + pi.off[rec2_b], page + pi.off[rec2_b], pi.size[rec2_b], cudaMemcpyHostToDevice,
		                    hp->in) != cudaSuccess) {
			return FLS_ERR_CUDA;
		}
		uint8_t* rb = nullptr;
		rc          = rec_decode(dp + pi.off[rec2_b], page + pi.off[rec2_b], pi.size[rec2_b], 2u, &rb, &rec2_n, hp->in);
		d_rec2.p    = rb;
		if (rc != FLS_OK) { return rc; }
	}
	ColDesc c {};
	rc = build_page_column(pi, dp, w, nullptr, 0, FLS_ORIGINAL, d_out.as<uint8_t>(), &c, d_rec.as<uint8_t>(), rec_n,
	                       d_rec2.as<uint8_t>(), rec2_n);
	if (rc != FLS_OK) { return rc; }
	auto ep = [&](uint32_t v, uint32_t b) -> uint64_t {
		if (v == 0) { return 0; }
		uint32_t x;
		std::memcpy(&x, page + pi.ep_off + 4ull * ((v - 1) * pi.arr_c + b), 4);
		return x;
	};
	// chunks of about 16 MB of output (fewer, larger copies: with both directions busy the link moves more in
	// long copies), the first of about 1 MB so that the copies out start early
	const uint64_t         chunk_vec = std::max<uint64_t>(1, (16ull << 20) / (1024 * sz));
	const uint64_t         first_vec = std::max<uint64_t>(1, (1ull << 20) / (1024 * sz));
	// chunk sizes double from the first up to the steady size, so that each chunk's copy in is done before the
	// copies out ahead of it are (a 1 MB chunk then a 16 MB one left the copies out idle while it came in)
	std::vector<uint32_t> bounds {0};
	uint64_t              step = first_vec;
	while (bounds.back() < pi.vec_c) {
		bounds.push_back(static_cast<uint32_t>(std::min<uint64_t>(pi.vec_c, bounds.back() + step)));
		step = std::min<uint64_t>(2 * step, chunk_vec);
	}
	const uint32_t n_chunks = static_cast<uint32_t>(bounds.size() - 1);
	if (3ull * n_chunks > kPipeEvents) { return FLS_ERR_TOO_LARGE; }
	cudaEvent_t* ev = hp->ev;
	const Family fam = post_is_patch(pi.layout->post)    ? Family::NUM_PATCH
	                   : !post_is_gather(pi.layout->post) ? Family::NUM
	                   : c.e <= 4                         ? Family::GATHER_NARROW
	                                                      : Family::GATHER;
	// page header, buffer offsets and entry points first, then every buffer but the largest whole (a few bytes
	// per vector: bit widths, bases, run counts), so that each chunk is one copy of the largest buffer's slice
	if (cudaMemcpyAsync(dp, page, pi.meta_sz, cudaMemcpyHostToDevice, hp->in) != cudaSuccess) { return FLS_ERR_CUDA; }
	int big = -1;
	for (uint32_t b = 0; b < pi.arr_c; ++b) {
		if (static_cast<int>(b) != rec_b && (big < 0 || pi.size[b] > pi.size[big])) { big = static_cast<int>(b); }
	}
	for (uint32_t b = 0; b < pi.arr_c; ++b) {
		if (static_cast<int>(b) == rec_b || static_cast<int>(b) == big || pi.size[b] == 0) { continue; }
		if (pi.off[b] + pi.size[b] <= page_size &&
		    cudaMemcpyAsync(dp + pi.off[b], page + pi.off[b], pi.size[b], cudaMemcpyHostToDevice, hp->in) != cudaSuccess) {
			return FLS_ERR_CUDA;
		}
	}
	for (uint32_t k = 0; k < n_chunks; ++k) {
		const uint32_t v0 = bounds[k];
		const uint32_t v1 = bounds[k + 1];
		if (k >= kPipeLead && cudaStreamWaitEvent(hp->in, ev[3 * (k - kPipeLead) + 2], 0) != cudaSuccess) {
			return FLS_ERR_CUDA;
		}
		for (uint32_t b = 0; b < pi.arr_c; ++b) {
			if (static_cast<int>(b) != big) { continue; } // the others are in place (rec buffers also decoded)
			const uint64_t lo = pi.off[b] + ep(v0, b);
			const uint64_t hi = v1 < pi.vec_c ? pi.off[b] + ep(v1, b) : pi.off[b] + pi.size[b];
			if (hi > lo && hi <= page_size &&
			    cudaMemcpyAsync(dp + lo, page + lo, hi - lo, cudaMemcpyHostToDevice, hp->in) != cudaSuccess) {
				return FLS_ERR_CUDA;
			}
		}
		if (cudaEventRecord(ev[3 * k], hp->in) != cudaSuccess || cudaStreamWaitEvent(hp->dec, ev[3 * k], 0) != cudaSuccess) {
			return FLS_ERR_CUDA;
		}
		DecodeArgs a {};
		a.col0      = c;
		a.queue     = hp->ids + v0;
		a.n_items   = v1 - v0;
		a.col_shift = 16;
		if (launch_decode(fam, a, hp->dec) != cudaSuccess) { return FLS_ERR_CUDA; }
		if (cudaEventRecord(ev[3 * k + 1], hp->dec) != cudaSuccess ||
		    cudaStreamWaitEvent(hp->out, ev[3 * k + 1], 0) != cudaSuccess) {
			return FLS_ERR_CUDA;
		}
		const uint64_t o0 = static_cast<uint64_t>(v0) * 1024 * sz, ob = static_cast<uint64_t>(v1 - v0) * 1024 * sz;
		if (cudaMemcpyAsync(static_cast<uint8_t*>(out) + o0, d_out.as<uint8_t>() + o0, ob, cudaMemcpyDeviceToHost,
		                    hp->out) != cudaSuccess ||
		    cudaEventRecord(ev[3 * k + 2], hp->out) != cudaSuccess) {
			return FLS_ERR_CUDA;
		}
	}
	// the buffers are freed on the copy-in stream: order it after the copies out
	const bool ok = cudaEventRecord(ev[0], hp->out) == cudaSuccess && cudaStreamWaitEvent(hp->in, ev[0], 0) == cudaSuccess &&
	                cudaStreamSynchronize(hp->out) == cudaSuccess;
	return ok ? FLS_OK : FLS_ERR_CUDA;
}

} // namespace
} // namespace flsgpu

using namespace flsgpu;

extern "C" {

connection_cpi* fls_cpi_connection_open() { return new Connection(); }

void fls_cpi_connection_close(connection_cpi* c) { delete c; }

int fls_encode_from_memory_status(void* in, uint64_t n, uint64_t cap, uint8_t* out, uint64_t* out_size,
                                  uint64_t* mtd_size, enum data_t dt, uint8_t expr) {
	if (!in && n >= 1024) { return FLS_ERR_ARG; }
	if (expr == 6) { // RLE DELTA_NO_PATCH
		const int w = value_width_of(dt);
		if (w != 32 && w != 64) { return FLS_ERR_UNSUPPORTED; }
		return encode_rle_page(in, n, cap, out, out_size, mtd_size, w);
	}
	switch (dt) {
	case INT64: return encode_t(static_cast<const uint64_t*>(in), n, cap, out, out_size, mtd_size, true, expr);
	case UINT64: return encode_t(static_cast<const uint64_t*>(in), n, cap, out, out_size, mtd_size, false, expr);
	case INT32: return encode_t(static_cast<const uint32_t*>(in), n, cap, out, out_size, mtd_size, true, expr);
	case UINT32: return encode_t(static_cast<const uint32_t*>(in), n, cap, out, out_size, mtd_size, false, expr);
	case DOUBLE:
		// the double pool's UNCOMPRESSED (src/cor/exp_pool.cpp:107): the values' bit patterns, transposed
		if (expr != 0) { return FLS_ERR_UNSUPPORTED; }
		return encode_t(static_cast<const uint64_t*>(in), n, cap, out, out_size, mtd_size, false, expr);
	default: return FLS_ERR_UNSUPPORTED;
	}
}

bool encode_from_memory(void* in, uint64_t n, uint64_t cap, uint8_t* out, uint64_t* out_size, uint64_t* mtd_size,
                        enum data_t dt, uint8_t expr) {
	return fls_encode_from_memory_status(in, n, cap, out, out_size, mtd_size, dt, expr) == FLS_OK;
}

int fls_decode_to_memory_checked(const uint8_t* enc, uint64_t enc_size, void* out, uint64_t out_cap, enum data_t dt,
                                 uint64_t* n_values) {
	return decode_host_page(enc, enc_size, out, out_cap, dt, n_values);
}

void decode_to_memory(uint8_t* enc, void* out, enum data_t dt) {
	// The reference API passes no sizes: the page size is derived from its own metadata and the caller
	// provides room for vec_c * 1024 values, as with the reference.
	(void)decode_host_page(enc, 0, out, ~0ull, dt, nullptr);
}

// init_random_access / random_access (include/fastlanes.h:88-108 of the reference, declared there and defined
// nowhere).  They serve the pages whose buffers are all per vector -- the C API's own expressions (UNCOMPRESSED,
// FFOR, DELTA, RLE, patched FFOR / DELTA without rec buffers) -- of INT64 columns (the functions carry no type).
// The byte range of buffer i of vector v is [off[i] + ep(v, i), off[i] + ep(v + 1, i)); the last vector's
// ranges end at the next buffer's offset, and its packed buffer at the page end, which the metadata alone does
// not give: init_random_access reports the largest packed vector there (64 * 128 bytes) and random_access takes
// the exact size from the vector's bit-width byte.
static const ExprLayout* random_access_layout(const uint8_t* page, PageInfo* pi) {
	if (!page || parse_page_header(page, 8 + 4 * 6, pi) != FLS_OK) { return nullptr; }
	const ExprLayout* L = pi->layout;
	if (L->ib_rec != kNoBuf || L->ib_rec2 != kNoBuf || L->post == POST_DICT || L->post == POST_RLE_DICT) {
		return nullptr;
	}
	return L;
}

static uint64_t ep_at(const uint8_t* page, const PageInfo& pi, uint64_t v, uint32_t i) {
	if (v == 0) { return 0; }
	uint32_t x;
	std::memcpy(&x, page + pi.ep_off + 4ull * ((v - 1) * pi.arr_c + i), 4);
	return x;
}

static constexpr uint64_t kMaxPackedVector = 64 * 128;

int fls_random_access_ranges(const uint8_t* page, uint64_t v, uint64_t* n_buf, uint64_t* pairs) {
	PageInfo          pi;
	const ExprLayout* L = random_access_layout(page, &pi);
	if (!L) { return FLS_ERR_UNSUPPORTED; }
	if (!n_buf || !pairs || v >= pi.vec_c) { return FLS_ERR_ARG; }
	*n_buf = pi.arr_c;
	for (uint32_t i = 0; i < pi.arr_c; ++i) {
		const uint64_t start = pi.off[i] + ep_at(page, pi, v, i);
		uint64_t       end;
		if (v + 1 < pi.vec_c) {
			end = pi.off[i] + ep_at(page, pi, v + 1, i);
		} else {
			end = i + 1 < pi.arr_c ? pi.off[i + 1] : start + kMaxPackedVector;
		}
		if (end < start) { return FLS_ERR_FORMAT; }
		pairs[2 * i]     = start;
		pairs[2 * i + 1] = end - start;
	}
	return FLS_OK;
}

int fls_random_access_decode(const uint8_t* page, uint64_t v, uint64_t n_buf, const uint64_t* pairs,
                             const uint8_t* const* buffers, int64_t* out) {
	PageInfo          pi;
	const ExprLayout* L = random_access_layout(page, &pi);
	if (!L) { return FLS_ERR_UNSUPPORTED; }
	if (!pairs || !buffers || !out || v >= pi.vec_c || n_buf != pi.arr_c) { return FLS_ERR_ARG; }
	// a one-vector page of the same expression: header with vec_c = 1, the buffer offsets, the vector's slices
	uint64_t size[6];
	uint64_t total = 8 + 4ull * pi.arr_c;
	for (uint32_t i = 0; i < pi.arr_c; ++i) {
		if (!buffers[i]) { return FLS_ERR_ARG; }
		size[i] = pairs[2 * i + 1];
	}
	const uint32_t last = pi.arr_c - 1;
	const uint64_t ws   = L->ws ? L->ws : 64;
	if (L->enc == ENC_RAW) {
		size[last] = ws * 128;
	} else {
		if (size[L->ib_bw] < 1) { return FLS_ERR_FORMAT; }
		const uint64_t bw = buffers[L->ib_bw][0];
		if (bw > ws) { return FLS_ERR_BW; }
		size[last] = bw * 128;
	}
	if (size[last] > pairs[2 * last + 1]) { return FLS_ERR_FORMAT; }
	for (uint32_t i = 0; i < pi.arr_c; ++i) { total += size[i]; }
	std::vector<uint8_t> one(total);
	std::memcpy(one.data(), page, 8);
	const uint16_t one_vec = 1;
	std::memcpy(one.data() + 4, &one_vec, 2);
	uint64_t pos = 8 + 4ull * pi.arr_c;
	for (uint32_t i = 0; i < pi.arr_c; ++i) {
		const uint32_t o = static_cast<uint32_t>(pos);
		std::memcpy(one.data() + 8 + 4 * i, &o, 4);
		if (size[i]) { std::memcpy(one.data() + pos, buffers[i], size[i]); }
		pos += size[i];
	}
	return decode_host_page(one.data(), total, out, 1024 * sizeof(int64_t), INT64, nullptr);
}

void init_random_access(uint8_t* in_encoded_data, uint64_t in_vector_id, uint64_t* output_n_buffer,
                        uint64_t* output_buffer) {
	if (fls_random_access_ranges(in_encoded_data, in_vector_id, output_n_buffer, output_buffer) != FLS_OK &&
	    output_n_buffer) {
		*output_n_buffer = 0;
	}
}

void random_access(uint8_t* in_encoded_data, uint64_t in_vector_id, uint64_t* output_n_buffer,
                   uint64_t* output_pair_offset_and_size, uint8_t** output_buffers, uint8_t* out_deencoded_vector) {
	(void)fls_random_access_decode(in_encoded_data, in_vector_id, output_n_buffer ? *output_n_buffer : 0,
	                               output_pair_offset_and_size, output_buffers,
	                               reinterpret_cast<int64_t*>(out_deencoded_vector));
}

int fls_page_placement(const uint8_t* page_prefix, uint64_t prefix_size, uint32_t* shift) {
	PageInfo pi;
	const int rc = parse_page_header(page_prefix, prefix_size, &pi);
	if (rc != FLS_OK) { return rc; }
	if (shift) { *shift = static_cast<uint32_t>((16 - pi.off[pi.layout->ib_packed] % 16) % 16); }
	return FLS_OK;
}

} // extern "C"
