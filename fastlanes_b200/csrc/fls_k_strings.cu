// String column kernels (see fls_strings.cuh for the formats).
//
//   k_fsst_dict      one CTA decodes a whole FSST-compressed dictionary: block scans of compressed and decoded
//                    lengths, then every entry decodes into place; writes cumulative END offsets (UNFSST).
//   k_str_lengths    warp per vector: the vector's 1024 codes (or row end offsets) in original order, the
//                    decoded length of every row, the vector total.
//   k_scan_totals    exclusive scan of the vector totals (one CTA): the first output byte of every vector.
//   k_str_materialize warp per vector: Arrow offsets of its rows and their bytes.  DICT rows are gathered from
//                    the decoded dictionary (held in shared memory when it fits) in aligned 16-byte output
//                    chunks; FSST / BYTE_ARR rows decode straight from the page.
#include "fls_decode.cu"
#include "fls_strings.cuh"
#include "fls_runtime.h"
#include "fls_strplan.h"
#include "fls_b200.h"

#include <cstring>
#include <mutex>

namespace flsgpu {

// ---------------------------------------------------------------------------------------------------------
// Block-wide exclusive scan of one value per thread (blockDim.x = 1024); returns the block total.
// ---------------------------------------------------------------------------------------------------------
template <class T>
__device__ __forceinline__ T block_exclusive_scan(T x, T* warp_tot, T* excl_out) {
	const uint32_t lane = threadIdx.x & 31u, warp = threadIdx.x >> 5;
	const T        inc  = warp_inclusive_scan(x, lane);
	if (lane == 31) { warp_tot[warp] = inc; }
	__syncthreads();
	if (warp == 0) {
		const T w  = lane < blockDim.x / 32 ? warp_tot[lane] : T(0);
		const T wi = warp_inclusive_scan(w, lane);
		warp_tot[lane] = wi - w; // exclusive per warp
		if (lane == 31) { warp_tot[32] = wi; }
	}
	__syncthreads();
	*excl_out     = warp_tot[warp] + inc - x;
	const T total = warp_tot[32];
	__syncthreads();
	return total;
}

__global__ void __launch_bounds__(1024) k_fsst_dict(const uint8_t* lens, const uint8_t* comp, uint64_t comp_size,
                                                    uint32_t entry_c, const FsstTable* tab, uint32_t* ends,
                                                    uint8_t* bytes, uint64_t bytes_cap, int* status) {
	__shared__ uint64_t sym[256];
	__shared__ uint8_t  len[256];
	__shared__ uint64_t wt[33];
	for (uint32_t i = threadIdx.x; i < 256; i += blockDim.x) {
		sym[i] = tab->sym[i];
		len[i] = tab->len[i];
	}
	__syncthreads();
	uint64_t ccarry = 0, dcarry = 0;
	bool     bad    = false;
	for (uint32_t base = 0; base < entry_c; base += blockDim.x) {
		const uint32_t i    = base + threadIdx.x;
		const uint64_t clen = i < entry_c ? ld_le(lens + 4ull * i, 4) : 0;
		uint64_t       cex;
		const uint64_t ctot = block_exclusive_scan<uint64_t>(clen, wt, &cex);
		const uint64_t coff = ccarry + cex;
		uint64_t       dlen = 0;
		const bool     in   = i < entry_c && coff + clen <= comp_size;
		bad |= i < entry_c && !in;
		if (in) { dlen = fsst_decoded_len(len, comp + coff, static_cast<uint32_t>(clen)); }
		uint64_t       dex;
		const uint64_t dtot = block_exclusive_scan<uint64_t>(dlen, wt, &dex);
		const uint64_t doff = dcarry + dex;
		if (in && doff + dlen <= bytes_cap) {
			fsst_decode_to(sym, len, comp + coff, static_cast<uint32_t>(clen), bytes + doff);
		} else if (in) {
			bad = true;
		}
		if (i < entry_c) { ends[i] = static_cast<uint32_t>(doff + dlen); }
		ccarry += ctot;
		dcarry += dtot;
	}
	if (bad) { atomicOr(status, STATUS_BAD_LAYOUT); }
}

// ---------------------------------------------------------------------------------------------------------
// Per-vector building blocks
// ---------------------------------------------------------------------------------------------------------
// Warp copy of n bytes global -> shared (16-byte loads when both sides allow it).
__device__ __forceinline__ void warp_copy(uint8_t* __restrict__ dst, const uint8_t* __restrict__ src, uint32_t n,
                                          uint32_t lane) {
	const uintptr_t al = reinterpret_cast<uintptr_t>(src) | reinterpret_cast<uintptr_t>(dst);
	if ((al & 15u) == 0) {
#pragma unroll 4
		for (uint32_t i = lane * 16; i + 16 <= n; i += 512) {
			*reinterpret_cast<uint4*>(dst + i) = __ldg(reinterpret_cast<const uint4*>(src + i));
		}
		for (uint32_t i = (n & ~15u) + lane; i < n; i += 32) { dst[i] = src[i]; }
	} else if ((al & 3u) == 0) {
#pragma unroll 8
		for (uint32_t i = lane * 4; i + 4 <= n; i += 128) {
			*reinterpret_cast<uint32_t*>(dst + i) = __ldg(reinterpret_cast<const uint32_t*>(src + i));
		}
		for (uint32_t i = (n & ~3u) + lane; i < n; i += 32) { dst[i] = src[i]; }
	} else {
#pragma unroll 8
		for (uint32_t i = lane; i < n; i += 32) { dst[i] = __ldg(src + i); }
	}
}

// The 1024 codes (DICT / DICT_RLE) or row end offsets (FSST / BYTE_ARR) of vector v, in ORIGINAL order, into
// rows[1024].  stage: >= 4096 + 128 bytes, gstage: >= 4096 + 32 bytes (RLE run values window).
__device__ bool load_rows(const ColDesc& c, uint32_t v, uint8_t* stage, uint8_t* gstage, uint32_t* rows,
                          uint32_t lane, int* status) {
	const Plan p = make_plan(c, v);
	if (!p.ok) {
		if (lane == 0) { atomicOr(status, p.bw > p.ws ? STATUS_BAD_BW : STATUS_BAD_LAYOUT); }
		return false;
	}
	warp_copy(stage, p.src, p.bytes, lane);
	if (p.post == POST_RLE && p.gbytes) { warp_copy(gstage, p.gsrc, p.gbytes, lane); }
	__syncwarp();
	bool bad = false;
	if (p.ws == 32) {
		uint32_t x[32];
		decode_stream<32>(p, reinterpret_cast<const uint32_t*>(stage), lane, x);
		const uint32_t r0 = run_start<32>(lane, 0);
#pragma unroll
		for (int i = 0; i < 32; ++i) { rows[r0 + i] = x[i]; }
	} else {
		uint32_t x[32];
		decode_stream<16>(p, reinterpret_cast<const uint32_t*>(stage), lane, x);
#pragma unroll
		for (int r = 0; r < 2; ++r) {
			const uint32_t r0 = run_start<16>(lane, r);
#pragma unroll
			for (int i = 0; i < 16; ++i) {
				const uint32_t idx = x[16 * r + i];
				const bool     in  = idx < p.n_runs;
				bad |= !in;
				rows[r0 + i] = in ? static_cast<uint32_t>(ld_le(gstage + 4ull * idx, 4)) : 0u;
			}
		}
	}
	if (__any_sync(0xFFFFFFFFu, bad) && lane == 0) { atomicOr(status, STATUS_BAD_INDEX); }
	__syncwarp();
	return true;
}

__device__ __forceinline__ uint32_t dict_start(const uint32_t* ends, uint32_t code) {
	return code == 0 ? 0u : ends[code - 1];
}

// Decoded length of row r of the vector (rows[] holds codes or end offsets in original order).
__device__ __forceinline__ uint32_t row_len(const StrArgs& a, const uint32_t* rows, uint32_t r, const uint8_t* vbytes,
                                            uint32_t vbytes_n, const uint8_t* flen, bool* bad) {
	if (a.kind == STR_DICT) {
		const uint32_t code = rows[r];
		if (code >= a.entry_c) {
			*bad = true;
			return 0;
		}
		return a.dict_ends[code] - dict_start(a.dict_ends, code);
	}
	const uint32_t s = r == 0 ? 0u : rows[r - 1];
	const uint32_t e = rows[r];
	if (e < s || e > vbytes_n) {
		*bad = true;
		return 0;
	}
	return a.kind == STR_BYTES ? e - s : fsst_decoded_len(flen, vbytes + s, e - s);
}

// bytes of vector v's compressed rows (FSST / BYTE_ARR): buffer 0 of the page at the vector's entry point
__device__ __forceinline__ const uint8_t* vector_bytes(const ColDesc& c, uint32_t v, uint32_t* n) {
	const uint32_t o   = ep_of(c, v, 0);
	const uint64_t end = (v + 1 < c.n_vec) ? ep_of(c, v + 1, 0) : c.buf_size[0];
	// a range outside the bytes buffer (corrupt entry points) leaves the vector with no bytes: every row with a
	// non-zero end offset is then reported as out of range
	*n = (end >= o && end <= c.buf_size[0]) ? static_cast<uint32_t>(end - o) : 0u;
	return *n ? c.buf[0] + o : c.buf[0];
}

constexpr int kStrWarps = 6;
constexpr int kStrWarpSmem = 4096 + 128 + 4096 + 32 + 4096 + 4100 + 12; // stage, gstage, rows, rel

struct StrWarpSmem {
	uint8_t*  stage;
	uint8_t*  gstage;
	uint32_t* rows;
	uint32_t* rel;
};

__device__ __forceinline__ StrWarpSmem str_warp_smem(uint8_t* base, uint32_t warp) {
	uint8_t*    w = base + warp * ((kStrWarpSmem + 15) & ~15);
	StrWarpSmem s;
	s.stage  = w;
	s.gstage = w + 4096 + 128;
	s.rows   = reinterpret_cast<uint32_t*>(w + 4096 + 128 + 4096 + 32);
	s.rel    = reinterpret_cast<uint32_t*>(w + 4096 + 128 + 4096 + 32 + 4096);
	return s;
}

__global__ void __launch_bounds__(kStrWarps * 32) k_str_lengths(const StrArgs a) {
	extern __shared__ __align__(128) uint8_t smem[];
	__shared__ uint8_t flen[256];
	if (a.kind == STR_FSST) {
		for (uint32_t i = threadIdx.x; i < 256; i += blockDim.x) { flen[i] = a.table->len[i]; }
	}
	__syncthreads();
	const uint32_t    lane = threadIdx.x & 31u, warp = threadIdx.x >> 5;
	const StrWarpSmem s    = str_warp_smem(smem, warp);
	const uint64_t    nw   = static_cast<uint64_t>(gridDim.x) * kStrWarps;
	for (uint64_t v = static_cast<uint64_t>(blockIdx.x) * kStrWarps + warp; v < a.col.n_vec; v += nw) {
		if (!load_rows(a.col, static_cast<uint32_t>(v), s.stage, s.gstage, s.rows, lane, a.status)) {
			if (lane == 0) { a.vec_total[v] = 0; }
			continue;
		}
		uint32_t       vn = 0;
		const uint8_t* vb = a.kind == STR_DICT ? nullptr : vector_bytes(a.col, static_cast<uint32_t>(v), &vn);
		bool           bad = false;
		uint64_t       sum = 0;
		for (uint32_t r = lane; r < kVec; r += 32) { sum += row_len(a, s.rows, r, vb, vn, flen, &bad); }
		sum = warp_sum(sum);
		if (__any_sync(0xFFFFFFFFu, bad) && lane == 0) { atomicOr(a.status, STATUS_BAD_INDEX); }
		if (lane == 0) { a.vec_total[v] = sum; }
		__syncwarp();
	}
}

__global__ void __launch_bounds__(1024) k_scan_totals(const uint64_t* total, uint64_t* base, uint64_t n) {
	__shared__ uint64_t wt[33];
	uint64_t            carry = 0;
	for (uint64_t b = 0; b < n; b += blockDim.x) {
		const uint64_t i = b + threadIdx.x;
		const uint64_t x = i < n ? total[i] : 0;
		uint64_t       ex;
		const uint64_t t = block_exclusive_scan<uint64_t>(x, wt, &ex);
		if (i < n) { base[i] = carry + ex; }
		carry += t;
	}
	if (threadIdx.x == 0) { base[n] = carry; }
}

__global__ void __launch_bounds__(kStrWarps * 32) k_str_materialize(const StrArgs a) {
	extern __shared__ __align__(128) uint8_t smem[];
	__shared__ uint64_t fsym[256];
	__shared__ uint8_t  flen[256];
	const uint32_t lane = threadIdx.x & 31u, warp = threadIdx.x >> 5;
	uint8_t*       dict_smem = smem + kStrWarps * ((kStrWarpSmem + 15) & ~15);
	// dictionary (bytes, then end offsets) into shared memory when the plan found room for it
	const uint8_t*  dbytes = a.dict_bytes;
	const uint32_t* dends  = a.dict_ends;
	if (a.kind == STR_DICT && a.dict_in_smem) {
		uint8_t* db = dict_smem;
		uint32_t* de = reinterpret_cast<uint32_t*>(dict_smem + ((a.dict_bytes_n + 15) & ~15ull));
		// the decoded dictionary lives in cudaMalloc'd (256-byte aligned) plan buffers
		const uint32_t nb16 = static_cast<uint32_t>((a.dict_bytes_n + 15) / 16);
		for (uint32_t i = threadIdx.x; i < nb16; i += blockDim.x) {
			reinterpret_cast<uint4*>(db)[i] = __ldg(reinterpret_cast<const uint4*>(a.dict_bytes) + i);
		}
		for (uint32_t i = threadIdx.x; i < a.entry_c; i += blockDim.x) { de[i] = __ldg(a.dict_ends + i); }
		dbytes = db;
		dends  = de;
	}
	if (a.kind == STR_FSST) {
		for (uint32_t i = threadIdx.x; i < 256; i += blockDim.x) {
			fsym[i] = a.table->sym[i];
			flen[i] = a.table->len[i];
		}
	}
	__syncthreads();
	StrArgs la = a;
	la.dict_ends = dends;
	const StrWarpSmem s  = str_warp_smem(smem, warp);
	const uint64_t    nw = static_cast<uint64_t>(gridDim.x) * kStrWarps;
	for (uint64_t v = static_cast<uint64_t>(blockIdx.x) * kStrWarps + warp; v < a.col.n_vec; v += nw) {
		const uint64_t vbase = a.vec_base[v];
		if (!load_rows(a.col, static_cast<uint32_t>(v), s.stage, s.gstage, s.rows, lane, a.status)) { continue; }
		uint32_t       vn = 0;
		const uint8_t* vb = a.kind == STR_DICT ? nullptr : vector_bytes(a.col, static_cast<uint32_t>(v), &vn);
		// row lengths of rows 32*lane .. 32*lane+31 (contiguous), local exclusive prefix, warp scan
		bool     bad = false;
		uint32_t run = 0;
		for (uint32_t i = 0; i < 32; ++i) {
			const uint32_t r = 32 * lane + i;
			s.rel[r]         = run;
			run += row_len(la, s.rows, r, vb, vn, flen, &bad);
		}
		const uint32_t inc = warp_inclusive_scan(run, lane);
		const uint32_t exc = inc - run;
		for (uint32_t i = 0; i < 32; ++i) { s.rel[32 * lane + i] += exc; }
		if (lane == 31) { s.rel[kVec] = inc; }
		if (__any_sync(0xFFFFFFFFu, bad) && lane == 0) { atomicOr(a.status, STATUS_BAD_INDEX); }
		__syncwarp();
		// Arrow offsets (u32) of the vector's rows, coalesced
		for (uint32_t r = lane; r < kVec; r += 32) {
			a.offsets[v * kVec + r] = static_cast<uint32_t>(vbase + s.rel[r]);
		}
		const uint32_t total = s.rel[kVec];
		if (v + 1 == a.col.n_vec && lane == 0) { a.offsets[(v + 1) * kVec] = static_cast<uint32_t>(vbase + total); }
		if (vbase + total > a.bytes_cap) {
			if (lane == 0) { atomicOr(a.status, STATUS_BAD_LAYOUT); }
			__syncwarp();
			continue;
		}
		if (a.kind == STR_DICT) {
			// 16-byte output chunks aligned in the output buffer; chunks shared with the neighbouring vectors are
			// written bytewise, the others with one 16-byte store
			const uint64_t b0 = vbase, b1 = vbase + total;
			const uint64_t q0 = b0 >> 4, q1 = (b1 + 15) >> 4;
			for (uint64_t q = q0 + lane; q < q1; q += 32) {
				const uint64_t lo = q * 16 > b0 ? q * 16 : b0;
				const uint64_t hi = q * 16 + 16 < b1 ? q * 16 + 16 : b1;
				uint32_t       rb = static_cast<uint32_t>(lo - b0);
				// last row whose start <= rb (skips empty rows)
				uint32_t l = 0, h = kVec;
				while (h - l > 1) {
					const uint32_t m = (l + h) >> 1;
					if (s.rel[m] <= rb) {
						l = m;
					} else {
						h = m;
					}
				}
				uint32_t r = l;
				uint32_t w[4] = {0u, 0u, 0u, 0u};
#pragma unroll
				for (uint32_t j = 0; j < 16; ++j) {
					const uint64_t b = q * 16 + j;
					if (b >= lo && b < hi) {
						const uint32_t rbj = static_cast<uint32_t>(b - b0);
						while (rbj >= s.rel[r + 1]) { ++r; }
						const uint32_t code = s.rows[r];
						w[j / 4] |= static_cast<uint32_t>(dbytes[dict_start(dends, code) + (rbj - s.rel[r])]) << (8 * (j % 4));
					}
				}
				uint8_t* dst = a.bytes + q * 16;
				if (lo == q * 16 && hi == q * 16 + 16) {
					*reinterpret_cast<uint4*>(dst) = make_uint4(w[0], w[1], w[2], w[3]);
				} else {
#pragma unroll
					for (uint32_t j = 0; j < 16; ++j) {
						const uint64_t b = q * 16 + j;
						if (b >= lo && b < hi) { dst[j] = static_cast<uint8_t>(w[j / 4] >> (8 * (j % 4))); }
					}
				}
			}
		} else {
			// FSST / BYTE_ARR: every lane decodes its 32 consecutive rows in place
			for (uint32_t i = 0; i < 32; ++i) {
				const uint32_t r  = 32 * lane + i;
				const uint32_t st = r == 0 ? 0u : s.rows[r - 1];
				const uint32_t en = s.rows[r];
				if (en < st || en > vn) { continue; }
				uint8_t* dst = a.bytes + vbase + s.rel[r];
				if (a.kind == STR_BYTES) {
					for (uint32_t b = 0; b < en - st; ++b) { dst[b] = vb[st + b]; }
				} else {
					fsst_decode_to(fsym, flen, vb + st, en - st, dst);
				}
			}
		}
		__syncwarp();
	}
}

// ---------------------------------------------------------------------------------------------------------
// Host launchers
// ---------------------------------------------------------------------------------------------------------
uint32_t str_smem_base() { return kStrWarps * ((kStrWarpSmem + 15) & ~15) + 64; }

cudaError_t launch_fsst_dict(const uint8_t* lens, const uint8_t* comp, uint64_t comp_size, uint32_t entry_c,
                             const FsstTable* tab, uint32_t* ends, uint8_t* bytes, uint64_t cap, int* status,
                             cudaStream_t s) {
	if (entry_c == 0) { return cudaSuccess; }
	k_fsst_dict<<<1, 1024, 0, s>>>(lens, comp, comp_size, entry_c, tab, ends, bytes, cap, status);
	++launch_counter();
	return cudaGetLastError();
}

cudaError_t launch_str_lengths(const StrArgs& a, int grid, cudaStream_t s) {
	const uint32_t smem = kStrWarps * ((kStrWarpSmem + 15) & ~15);
	static bool    set  = false;
	if (!set) {
		cudaFuncSetAttribute(k_str_lengths, cudaFuncAttributeMaxDynamicSharedMemorySize, smem);
		set = true;
	}
	k_str_lengths<<<grid, kStrWarps * 32, smem, s>>>(a);
	++launch_counter();
	return cudaGetLastError();
}

cudaError_t launch_scan_totals(const uint64_t* total, uint64_t* base, uint64_t n, cudaStream_t s) {
	k_scan_totals<<<1, 1024, 0, s>>>(total, base, n);
	++launch_counter();
	return cudaGetLastError();
}

cudaError_t launch_str_materialize(const StrArgs& a, int grid, uint32_t dyn_smem, cudaStream_t s) {
	static uint32_t set = 0;
	if (dyn_smem > set) {
		cudaError_t e = cudaFuncSetAttribute(k_str_materialize, cudaFuncAttributeMaxDynamicSharedMemorySize, dyn_smem);
		if (e != cudaSuccess) { return e; }
		set = dyn_smem;
	}
	k_str_materialize<<<grid, kStrWarps * 32, dyn_smem, s>>>(a);
	++launch_counter();
	return cudaGetLastError();
}

} // namespace flsgpu

// =========================================================================================================
// Allocation-free decode of FSST / BYTE_ARR string pages (fls_gpu_decode_fsst_page_noalloc).
//
// The string plan keeps its scratch (per-vector byte totals and first-byte bases, the FSST table, a status
// word) in cudaMalloc'd buffers.  This variant keeps the same scratch in one array compiled into the library,
// so the call allocates nothing; in exchange the page may hold at most kNoAllocMaxVectors vectors.
// =========================================================================================================
namespace flsgpu {

constexpr uint32_t kNoAllocMaxVectors = 8192; // 8,388,608 rows per call

struct NoAllocLayout {
	static constexpr size_t kStatus = 0;                                      // int, OR-ed device status
	static constexpr size_t kTable  = 256;                                    // FsstTable (2304 B)
	static constexpr size_t kTotal  = kTable + ((sizeof(FsstTable) + 255) & ~size_t(255));
	static constexpr size_t kBase   = kTotal + 8 * (kNoAllocMaxVectors + 1);
	static constexpr size_t kBytes  = kBase + 8 * (kNoAllocMaxVectors + 1);   // 133,376 B in all
};

// Every GPU that loads the library holds this array until the process exits.
static __device__ __align__(256) uint8_t g_noalloc_scratch[NoAllocLayout::kBytes];

// Device address of g_noalloc_scratch on the current device, looked up once per device on the first call.
static uint8_t* noalloc_scratch() {
	static uint8_t*   addr[64] = {};
	static std::mutex mu;
	int               dev      = 0;
	if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= 64) { return nullptr; }
	std::lock_guard<std::mutex> lk(mu);
	if (!addr[dev]) {
		void* p = nullptr;
		if (cudaGetSymbolAddress(&p, g_noalloc_scratch) != cudaSuccess || p == nullptr) { return nullptr; }
		addr[dev] = static_cast<uint8_t*>(p);
	}
	return addr[dev];
}

int fsst_import_table(const uint8_t* buf, uint64_t avail, FsstTable* t, uint64_t* used);

} // namespace flsgpu

extern "C" int fls_gpu_decode_fsst_page_noalloc(const uint8_t* d_page, uint64_t page_size, const uint8_t* d_dict,
                                                uint64_t dict_size, uint32_t* d_offsets, uint8_t* d_bytes,
                                                uint64_t bytes_cap, int* d_status, void* stream) {
	using namespace flsgpu;
	if (!d_page || !d_offsets || (!d_bytes && bytes_cap) || (reinterpret_cast<uintptr_t>(d_bytes) & 15u) != 0 ||
	    bytes_cap >= (1ull << 32)) {
		return FLS_ERR_ARG;
	}
	cudaStream_t s = static_cast<cudaStream_t>(stream);
	uint8_t      hdr[8 + 4 * 5];
	const uint64_t take = page_size < sizeof(hdr) ? page_size : sizeof(hdr);
	if (take < 8 || cudaMemcpy(hdr, d_page, take, cudaMemcpyDeviceToHost) != cudaSuccess) { return FLS_ERR_FORMAT; }
	uint8_t kind = 0, arr_c = 0, ws = 32, enc = ENC_RAW, ib_packed = 1, ib_bw = kNoBuf, ib_base = kNoBuf,
	        ib_lane = kNoBuf;
	if (hdr[0] == 7 && hdr[1] == 1) {
		kind = STR_FSST, arr_c = 2; // FSST: bytes, end offsets
	} else if (hdr[0] == 7 && hdr[1] == 2) {
		kind = STR_FSST, arr_c = 5, enc = ENC_DELTA, ib_packed = 4, ib_bw = 2, ib_base = 3, ib_lane = 1;
	} else if (hdr[0] == 3 && hdr[1] == 1) {
		kind = STR_BYTES, arr_c = 2; // BYTE_ARR: bytes, end offsets
	} else {
		return FLS_ERR_UNSUPPORTED;
	}
	uint16_t vec_c = 0;
	std::memcpy(&vec_c, hdr + 4, 2);
	if (vec_c > kNoAllocMaxVectors) { return FLS_ERR_TOO_LARGE; }
	if (take < 8ull + 4 * arr_c) { return FLS_ERR_FORMAT; }
	uint32_t off[5];
	for (uint32_t i = 0; i < arr_c; ++i) { std::memcpy(&off[i], hdr + 8 + 4 * i, 4); }
	const uint64_t meta = 8 + 4ull * arr_c + 4ull * arr_c * (vec_c ? vec_c - 1 : 0);
	ColDesc        c {};
	for (uint32_t i = 0; i < arr_c; ++i) {
		const uint64_t end = (i + 1 < arr_c) ? off[i + 1] : page_size;
		if (off[i] < meta || off[i] > end || end > page_size) { return FLS_ERR_FORMAT; }
		c.buf[i]      = d_page + off[i];
		c.buf_size[i] = end - off[i];
	}
	uint8_t* scratch = noalloc_scratch();
	if (!scratch) { return FLS_ERR_CUDA; }
	FsstTable tab {};
	if (kind == STR_FSST) {
		// dict_hdr_t followed by the exported symbol table (at most FSST_MAXHEADER = 2066 bytes)
		uint8_t        h[8 + 2066];
		const uint64_t n = dict_size < sizeof(h) ? dict_size : sizeof(h);
		if (!d_dict || n < 8 + 17 || cudaMemcpy(h, d_dict, n, cudaMemcpyDeviceToHost) != cudaSuccess) {
			return FLS_ERR_FORMAT;
		}
		const int rc = fsst_import_table(h + 8, n - 8, &tab, nullptr);
		if (rc != FLS_OK) { return rc; }
	}
	// the table and a zero status are the only scratch contents a call relies on; totals and bases are
	// rewritten in full by every call
	if (cudaMemcpyAsync(scratch + NoAllocLayout::kTable, &tab, sizeof(tab), cudaMemcpyHostToDevice, s) != cudaSuccess ||
	    cudaMemsetAsync(scratch + NoAllocLayout::kStatus, 0, sizeof(int), s) != cudaSuccess) {
		return FLS_ERR_CUDA;
	}
	c.ws            = ws;
	c.e             = 4;
	c.enc           = enc;
	c.post          = POST_NONE;
	c.order         = 1;
	c.layout        = LAYOUT_PAGE;
	c.arr_c         = arr_c;
	c.n_vec         = vec_c;
	c.ib_bw         = ib_bw;
	c.ib_base       = ib_base;
	c.ib_packed     = ib_packed;
	c.ib_lane_bases = ib_lane;
	c.ib_vals       = kNoBuf;
	c.ep            = reinterpret_cast<const uint32_t*>(d_page + 8 + 4 * arr_c);
	if (vec_c == 0) { return cudaMemsetAsync(d_offsets, 0, 4, s) == cudaSuccess ? FLS_OK : FLS_ERR_CUDA; }
	StrArgs a {};
	a.col       = c;
	a.kind      = kind;
	a.table     = reinterpret_cast<const FsstTable*>(scratch + NoAllocLayout::kTable);
	a.vec_total = reinterpret_cast<uint64_t*>(scratch + NoAllocLayout::kTotal);
	a.vec_base  = reinterpret_cast<const uint64_t*>(scratch + NoAllocLayout::kBase);
	a.offsets   = d_offsets;
	a.bytes     = d_bytes;
	a.bytes_cap = bytes_cap;
	a.status    = d_status ? d_status : reinterpret_cast<int*>(scratch + NoAllocLayout::kStatus);
	int sms = 0, dev = 0;
	if (cudaGetDevice(&dev) != cudaSuccess ||
	    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess || sms <= 0) {
		return FLS_ERR_CUDA;
	}
	if (launch_str_lengths(a, sms, s) != cudaSuccess ||
	    launch_scan_totals(a.vec_total, reinterpret_cast<uint64_t*>(scratch + NoAllocLayout::kBase), vec_c, s) !=
	        cudaSuccess ||
	    launch_str_materialize(a, sms, str_smem_base(), s) != cudaSuccess) {
		return FLS_ERR_CUDA;
	}
	return FLS_OK;
}
