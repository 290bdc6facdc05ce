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
__device__ __forceinline__ void warp_copy(uint8_t* dst, const uint8_t* src, uint32_t n, uint32_t lane) {
	if (((reinterpret_cast<uintptr_t>(src) | reinterpret_cast<uintptr_t>(dst)) & 15u) == 0) {
		for (uint32_t i = lane * 16; i + 16 <= n; i += 512) {
			*reinterpret_cast<uint4*>(dst + i) = *reinterpret_cast<const uint4*>(src + i);
		}
		for (uint32_t i = (n & ~15u) + lane; i < n; i += 32) { dst[i] = src[i]; }
	} else {
		for (uint32_t i = lane; i < n; i += 32) { dst[i] = src[i]; }
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
		for (uint32_t i = threadIdx.x; i < a.dict_bytes_n; i += blockDim.x) { db[i] = a.dict_bytes[i]; }
		for (uint32_t i = threadIdx.x; i < a.entry_c; i += blockDim.x) { de[i] = a.dict_ends[i]; }
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
				uint8_t  chunk[16];
				for (uint64_t b = lo; b < hi; ++b, ++rb) {
					while (rb >= s.rel[r + 1]) { ++r; }
					const uint32_t code = s.rows[r];
					chunk[b - q * 16]   = dbytes[dict_start(dends, code) + (rb - s.rel[r])];
				}
				uint8_t* dst = a.bytes + q * 16;
				if (lo == q * 16 && hi == q * 16 + 16) {
					uint4 x;
					memcpy(&x, chunk, 16);
					*reinterpret_cast<uint4*>(dst) = x;
				} else {
					for (uint64_t b = lo; b < hi; ++b) { dst[b - q * 16] = chunk[b - q * 16]; }
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
