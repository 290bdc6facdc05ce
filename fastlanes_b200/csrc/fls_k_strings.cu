// String column kernels (see fls_strings.cuh for the formats).
//
//   k_fsst_dict      one CTA decodes a whole FSST-compressed dictionary: block scans of compressed and decoded
//                    lengths, then every entry decodes into place; writes cumulative END offsets (UNFSST).
//   k_str_lengths    warp per vector: the vector's 1024 codes (or row end offsets) in original order, the
//                    decoded length of every row, the vector total.
//   k_scan_totals    exclusive scan of the vector totals (one CTA): the first output byte of every vector.
//   k_str_materialize warp per vector: Arrow offsets of its rows and their bytes, 32 rows at a time (one per
//                    lane) into a per-warp shared-memory window that leaves in coalesced 16-byte stores.  DICT
//                    rows are copied from the decoded dictionary (held in shared memory when it fits), BYTE_ARR
//                    rows from the page, FSST and FSST12 rows decode from the page (symbol table in shared
//                    memory: 2.3 KB for FSST, 36 KB for FSST12).
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
__device__ __forceinline__ uint32_t dict_start(const uint32_t* ends, uint32_t code) {
	return code == 0 ? 0u : ends[code - 1];
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

// ---------------------------------------------------------------------------------------------------------
// Per-warp shared memory of the string kernels (warps per CTA chosen at launch)
//   plans   the next kStrPB plans (64 B each) of the warp's vectors, fetched lane-parallel
//   rows    the vector's packed codes / end offsets (copied in, with 128 bytes of slack for the extraction),
//           then, once decoded, its 1024 codes / end offsets in original order (row r at word r + r / 32:
//           conflict-free both by run and by row).  Dictionaries of fewer than 65535 entries keep their codes
//           as 16-bit values (row r at half-word r + 2 * (r / 32), as conflict-free) in half the space: their
//           packed codes are at most 16 bits wide
//   window  (materialize only) 2 KB of output bytes starting at a 16-byte aligned output position; the copied
//           kinds (DICT, BYTE_ARR) store whole words (put_row), so only the partly filled word is kept zero
//           past the filled bytes
// The work per vector (1024 row copies) is long next to the latency of its loads, so the packed words are
// read synchronously: occupancy, not prefetch depth, is what hides latency here.
// ---------------------------------------------------------------------------------------------------------
constexpr uint32_t kStrPB      = 4;
constexpr uint32_t kStrRows    = 4096 + 128; // >= 1055 padded row words, >= 128 * (32 + 1) staged bytes
constexpr uint32_t kStrRows16  = 2048 + 128; // >= 1086 padded 16-bit rows, >= 128 * (16 + 1) staged bytes
constexpr uint32_t kStrWindow  = 2048;

enum : int { STR_PASS_LENGTHS = 0, STR_PASS_MATERIALIZE = 1 };

// per-warp shared memory of the single-pass FSST / BYTE_ARR kernel: rows, then the window (no plan ring)
constexpr uint32_t kStreamSinglePerWarp = kStrRows + kStrWindow;

__host__ __device__ constexpr uint32_t str_rows_bytes(bool r16) { return r16 ? kStrRows16 : kStrRows; }

__host__ __device__ constexpr uint32_t str_per_warp(int pass, bool r16) {
	return kStrPB * 64 + str_rows_bytes(r16) + (pass == STR_PASS_MATERIALIZE ? kStrWindow : 0u);
}

__device__ __forceinline__ uint32_t row_word(uint32_t r) { return r + (r >> 5); }
__device__ __forceinline__ uint32_t row_half(uint32_t r) { return r + 2 * (r >> 5); }

// row r of the decoded rows in buf (32- or 16-bit layout)
template <bool R16>
__device__ __forceinline__ uint32_t row_at(const uint8_t* buf, uint32_t r) {
	if constexpr (R16) {
		return reinterpret_cast<const uint16_t*>(buf)[row_half(r)];
	} else {
		return reinterpret_cast<const uint32_t*>(buf)[row_word(r)];
	}
}

template <bool R16>
__device__ __forceinline__ void set_row(uint8_t* buf, uint32_t r, uint32_t x) {
	if constexpr (R16) {
		// codes past 16 bits become 0xFFFF, which is out of range for every 16-bit dictionary
		reinterpret_cast<uint16_t*>(buf)[row_half(r)] = static_cast<uint16_t>(x < 0xFFFFu ? x : 0xFFFFu);
	} else {
		reinterpret_cast<uint32_t*>(buf)[row_word(r)] = x;
	}
}

// Codes (or end offsets) of the vector into rows in original order.  DICT_RLE run values are read from the
// page directly.  False (status set) when the packed codes do not fit the 16-bit layout's staging space.
template <bool R16>
__device__ __forceinline__ bool load_rows(const Plan& p, uint8_t* buf, uint32_t lane, int* status) {
	if (R16 && p.bytes + 128 > kStrRows16) {
		if (lane == 0) { atomicOr(status, STATUS_BAD_LAYOUT); }
		return false;
	}
	const uintptr_t al = reinterpret_cast<uintptr_t>(p.src);
	if ((al & 15u) == 0) {
		const uint4* s = reinterpret_cast<const uint4*>(p.src);
		uint4*       d = reinterpret_cast<uint4*>(buf);
		for (uint32_t i = lane; i < p.bytes / 16; i += 32) { d[i] = __ldg(s + i); }
	} else if ((al & 3u) == 0) {
		const uint32_t* s = reinterpret_cast<const uint32_t*>(p.src);
		uint32_t*       d = reinterpret_cast<uint32_t*>(buf);
		for (uint32_t i = lane; i < p.bytes / 4; i += 32) { d[i] = __ldg(s + i); }
	} else {
		for (uint32_t i = lane; i < p.bytes; i += 32) { buf[i] = __ldg(p.src + i); }
	}
	__syncwarp();
	uint32_t x[32];
	bool     bad = false;
	if (p.ws == 32) {
		decode_stream<32>(p, reinterpret_cast<const uint32_t*>(buf), lane, x);
		__syncwarp();
		const uint32_t r0 = run_start<32>(lane, 0);
#pragma unroll
		for (int i = 0; i < 32; ++i) { set_row<R16>(buf, r0 + i, x[i]); }
	} else {
		decode_stream<16>(p, reinterpret_cast<const uint32_t*>(buf), lane, x);
#pragma unroll
		for (int i = 0; i < 32; ++i) {
			const bool in = x[i] < p.n_runs;
			bad |= !in;
			x[i] = in ? static_cast<uint32_t>(ld_le(p.gsrc + 4ull * x[i], 4)) : 0u;
		}
		__syncwarp();
#pragma unroll
		for (int r = 0; r < 2; ++r) {
			const uint32_t r0 = run_start<16>(lane, r);
#pragma unroll
			for (int i = 0; i < 16; ++i) { set_row<R16>(buf, r0 + i, x[16 * r + i]); }
		}
	}
	if (__any_sync(0xFFFFFFFFu, bad) && lane == 0) { atomicOr(status, STATUS_BAD_INDEX); }
	__syncwarp();
	return true;
}

// Row r of the vector: its source (dictionary entry or compressed bytes) and decoded length.
struct RowRef {
	uint32_t start; // dictionary byte offset (DICT) or compressed byte offset within the vector
	uint32_t clen;  // compressed length (FSST / BYTE_ARR)
	uint32_t len;   // decoded length
};

template <int KIND, bool R16>
__device__ __forceinline__ RowRef row_ref(const StrArgs& a, const uint32_t* ends, const uint8_t* rows, uint32_t r,
                                          const uint8_t* vb, uint32_t vn, const uint8_t* flen, bool* bad,
                                          const uint32_t* packed = nullptr, const uint32_t* known_len = nullptr) {
	RowRef f {0, 0, 0};
	if constexpr (KIND == STR_DICT) {
		const uint32_t code = row_at<R16>(rows, r);
		if (code >= a.entry_c) {
			*bad = true;
			return f;
		}
		if (packed) {
			const uint32_t e = __ldg(packed + code);
			f.start          = e & 0xFFFFFFu;
			f.len            = e >> 24;
			return f;
		}
		f.start = code ? ends[code - 1] : 0u;
		f.len   = ends[code] - f.start;
		return f;
	} else {
		const uint32_t s = r == 0 ? 0u : row_at<R16>(rows, r - 1);
		const uint32_t e = row_at<R16>(rows, r);
		if (e < s || e > vn) {
			*bad = true;
			return f;
		}
		f.start = s;
		f.clen  = e - s;
		if constexpr (KIND == STR_BYTES) {
			f.len = f.clen;
		} else if (known_len) {
			f.len = known_len[r];
		} else if constexpr (KIND == STR_FSST12) {
			f.len = fsst12_decoded_len(flen, vb + s, f.clen);
		} else {
			f.len = fsst_decoded_len(flen, vb + s, f.clen);
		}
		return f;
	}
}


// One pass over the column's vectors, warp per vector.  LENGTHS: per-vector decoded byte totals.  MATERIALIZE:
// Arrow offsets and bytes, at the first output byte of every vector computed from the totals.  SM (DICT only):
// SM_ENDS (lengths pass) copies the dictionary end offsets to shared memory (after the per-warp areas) at CTA
// start, SM_BYTES (materialising pass) the decoded dictionary bytes.
enum : int { SM_NONE = 0, SM_ENDS = 1, SM_BYTES = 2 };

template <int PASS, int KIND, int SM, bool R16>
__global__ void __launch_bounds__(kStrMaxWarps * 32) k_str_pass(const StrArgs a) {
	extern __shared__ __align__(128) uint8_t smem[];
	constexpr uint32_t  kSyms = KIND == STR_FSST ? 256 : KIND == STR_FSST12 ? 4096 : 1;
	__shared__ uint64_t fsym[kSyms];
	__shared__ uint8_t  flen[kSyms];
	const uint32_t     lane = threadIdx.x & 31u, warp = threadIdx.x >> 5, nwarps = blockDim.x >> 5;
	constexpr uint32_t kPerWarp = str_per_warp(PASS, R16);
	const uint8_t*     dict     = a.dict_bytes;
	const uint32_t*    ends     = a.dict_ends;
	if constexpr (KIND == STR_DICT && (SM & SM_ENDS)) {
		uint32_t* es = reinterpret_cast<uint32_t*>(smem + nwarps * kPerWarp);
		for (uint32_t i = threadIdx.x; i < a.entry_c; i += blockDim.x) { es[i] = __ldg(a.dict_ends + i); }
		ends = es;
	}
	if constexpr (PASS == STR_PASS_MATERIALIZE && KIND == STR_DICT && SM == SM_BYTES) {
		uint8_t* db = smem + nwarps * kPerWarp;
		// the decoded dictionary lives in a cudaMalloc'd (256-byte aligned) buffer with at least 16 bytes of
		// slack after the last entry
		const uint32_t nb16 = static_cast<uint32_t>((a.dict_bytes_n + 15) / 16);
		for (uint32_t i = threadIdx.x; i < nb16; i += blockDim.x) {
			reinterpret_cast<uint4*>(db)[i] = __ldg(reinterpret_cast<const uint4*>(a.dict_bytes) + i);
		}
		dict = db;
	}
	if constexpr (KIND == STR_FSST) {
		for (uint32_t i = threadIdx.x; i < 256; i += blockDim.x) {
			fsym[i] = a.table->sym[i];
			flen[i] = a.table->len[i];
		}
	}
	if constexpr (KIND == STR_FSST12) {
		for (uint32_t i = threadIdx.x; i < 4096; i += blockDim.x) { fsym[i] = __ldg(a.table12->sym + i); }
		for (uint32_t i = threadIdx.x; i < 4096 / 16; i += blockDim.x) {
			reinterpret_cast<uint4*>(flen)[i] = __ldg(reinterpret_cast<const uint4*>(a.table12->len) + i);
		}
	}
	uint8_t* wbase = smem + warp * kPerWarp;
	PlanS*   plans = reinterpret_cast<PlanS*>(wbase);
	uint8_t* buf   = wbase + kStrPB * 64;
	uint8_t* win   = buf + str_rows_bytes(R16);
	// kOr: rows go to the window as whole words (put_row, fsst_put_row); FSST12 rows as bytes
	constexpr bool kOr  = PASS == STR_PASS_MATERIALIZE && KIND != STR_FSST12;
	uint32_t*      win32 = reinterpret_cast<uint32_t*>(win);
	__syncthreads();

	const uint64_t gw = static_cast<uint64_t>(blockIdx.x) * nwarps + warp;
	const uint64_t nw = static_cast<uint64_t>(gridDim.x) * nwarps;
	const uint64_t n  = a.col.n_vec;
	uint32_t       k  = 0;
	for (uint64_t v = gw; v < n; v += nw, ++k) {
		if (k % kStrPB == 0) {
			if (lane < kStrPB) {
				const uint64_t u = v + lane * nw;
				Plan           q {};
				if (u < n) { q = make_plan(a.col, static_cast<uint32_t>(u)); }
				plans[lane] = pack_plan(q, u < n);
			}
			__syncwarp();
		}
		const Plan p = unpack_plan(plans[k % kStrPB]);
		if (!p.ok) {
			if (lane == 0) {
				atomicOr(a.status, p.bw > p.ws ? STATUS_BAD_BW : STATUS_BAD_LAYOUT);
				if (PASS == STR_PASS_LENGTHS) { a.vec_total[v] = 0; }
			}
			continue;
		}
		if (!load_rows<R16>(p, buf, lane, a.status)) {
			if (PASS == STR_PASS_LENGTHS && lane == 0) { a.vec_total[v] = 0; }
			__syncwarp();
			continue;
		}
		const uint8_t* rows = buf;
		uint32_t        vn   = 0;
		const uint8_t*  vb   = KIND == STR_DICT ? nullptr : vector_bytes(a.col, static_cast<uint32_t>(v), &vn);
		bool            bad  = false;
		if constexpr (PASS == STR_PASS_LENGTHS) {
			uint32_t sum = 0;
			for (uint32_t b = 0; b < kVec / 32; ++b) {
				const uint32_t l = row_ref<KIND, R16>(a, ends, rows, 32 * b + lane, vb, vn, flen, &bad).len;
				if (KIND != STR_DICT && KIND != STR_BYTES && a.row_len) { a.row_len[v * kVec + 32 * b + lane] = l; }
				sum += l;
			}
			sum = warp_sum(sum);
			if (__any_sync(0xFFFFFFFFu, bad) && lane == 0) { atomicOr(a.status, STATUS_BAD_INDEX); }
			if (lane == 0) { a.vec_total[v] = sum; }
			__syncwarp();
			continue;
		} else {
			const uint64_t vbase = a.vec_base[v];
			const uint64_t vend  = a.vec_base[v + 1];
			if (vend < vbase || vend > a.bytes_cap) {
				if (lane == 0) { atomicOr(a.status, STATUS_BAD_LAYOUT); }
				__syncwarp();
				continue;
			}
			// Rows go to the window in batches of 32 (one row per lane, positions from a warp scan of the
			// lengths); full 16-byte chunks of the window go out with 16-byte stores, the vector's first and last
			// partial chunks byte by byte (the neighbouring vectors write the other bytes of those chunks).
			uint64_t W    = vbase & ~15ull; // output position of win[0]
			uint32_t fill = static_cast<uint32_t>(vbase & 15u);
			uint64_t lo   = vbase; // first output byte the window may write
			if constexpr (kOr) {
				// the first row may start inside this word: it ORs its bytes in
				if (lane == 0) { win32[fill >> 2] = 0; }
				__syncwarp();
			}
			auto flush = [&](bool all) {
				const uint32_t full = fill & ~15u;
				const uint32_t upto = all ? fill : full;
				for (uint32_t c = 16 * lane; c < upto; c += 512) {
					const uint64_t g = W + c;
					if (g >= lo && c + 16 <= upto) {
						*reinterpret_cast<uint4*>(a.bytes + g) = *reinterpret_cast<const uint4*>(win + c);
					} else {
						for (uint32_t i = 0; i < 16 && c + i < upto; ++i) {
							if (g + i >= lo) { a.bytes[g + i] = win[c + i]; }
						}
					}
				}
				__syncwarp();
				if (!all) {
					// the partial chunk [full, fill) moves to the window start
					if constexpr (kOr) {
						// (its bytes past `fill` are zero: every word was stored whole, zeros past the row's end)
						if (lane == 0 && full != 0 && (fill & 15u) != 0) {
							*reinterpret_cast<uint4*>(win) = *reinterpret_cast<const uint4*>(win + full);
						}
					} else {
						const uint8_t t = lane < (fill & 15u) ? win[full + lane] : 0;
						__syncwarp();
						if (lane < (fill & 15u)) { win[lane] = t; }
					}
					__syncwarp();
					W += full;
					fill &= 15u;
					lo = lo > W ? lo : W;
				}
			};
			uint32_t  vpos = 0; // bytes of this vector emitted so far
			uint32_t* offs = a.offsets + v * kVec + lane;
			// the next batch's row is looked up while the current one is copied
			const uint32_t* known = a.row_len ? a.row_len + v * kVec : nullptr;
			RowRef next = row_ref<KIND, R16>(a, ends, rows, lane, vb, vn, flen, &bad, a.dict_rows, known);
			for (uint32_t b = 0; b < kVec / 32; ++b) {
				const uint32_t r = 32 * b + lane;
				const RowRef   f = next;
				if (b + 1 < kVec / 32) {
					next = row_ref<KIND, R16>(a, ends, rows, r + 32, vb, vn, flen, &bad, a.dict_rows, known);
				}
				const uint32_t inc = warp_inclusive_scan(f.len, lane);
				const uint32_t o   = vpos + inc - f.len;
				const uint32_t T   = __shfl_sync(0xFFFFFFFFu, inc, 31);
				offs[32 * b] = static_cast<uint32_t>(vbase + o);
				if (fill + T > kStrWindow) { flush(false); }
				if (fill + T <= kStrWindow) {
					if constexpr (kOr) {
						uint32_t hk = 0, head = 0;
						bool     mid;
						if constexpr (KIND == STR_DICT) {
							// the decoded dictionary starts 16-byte aligned (shared or global memory)
							mid = put_row(win32, fill + (o - vpos), reinterpret_cast<const uint32_t*>(dict), f.start,
							              f.len, &hk, &head);
						} else if constexpr (KIND == STR_FSST) {
							mid = fsst_put_row(win32, fill + (o - vpos), fsym, flen, vb + f.start, f.clen, &hk, &head);
						} else {
							const uintptr_t va = reinterpret_cast<uintptr_t>(vb);
							mid = put_row(win32, fill + (o - vpos), reinterpret_cast<const uint32_t*>(va & ~uintptr_t(3)),
							              f.start + static_cast<uint32_t>(va & 3u), f.len, &hk, &head);
						}
						__syncwarp(); // every word's whole store lands before the rows that start inside it OR in
						if (mid) { atomicOr(win32 + hk, head); }
					} else {
						fsst12_decode_to(fsym, flen, vb + f.start, f.clen, win + fill + (o - vpos));
					}
					fill += T;
				} else {
					// a batch larger than the window: its rows go straight to global memory, after the window's
					// pending bytes
					flush(true);
					uint8_t* dst = a.bytes + vbase + o;
					if constexpr (KIND == STR_FSST) {
						fsst_decode_to(fsym, flen, vb + f.start, f.clen, dst);
					} else if constexpr (KIND == STR_FSST12) {
						fsst12_decode_to(fsym, flen, vb + f.start, f.clen, dst);
					} else {
						const uint8_t* src = KIND == STR_DICT ? dict + f.start : vb + f.start;
						for (uint32_t i = 0; i < f.len; ++i) { dst[i] = src[i]; }
					}
					const uint64_t pos = vbase + vpos + T;
					W    = pos & ~15ull;
					fill = static_cast<uint32_t>(pos & 15u);
					lo   = pos;
					if constexpr (kOr) {
						__syncwarp();
						if (lane == 0) { win32[fill >> 2] = 0; }
					}
				}
				vpos += T;
				__syncwarp();
			}
			flush(true);
			if (lane == 0 && v + 1 == n) { a.offsets[n * kVec] = static_cast<uint32_t>(vbase + vpos); }
			if (vbase + vpos != vend) { bad = true; }
			if (__any_sync(0xFFFFFFFFu, bad) && lane == 0) { atomicOr(a.status, STATUS_BAD_INDEX); }
			__syncwarp();
		}
	}
}

// One pass over an FSST or BYTE_ARR column, warp per vector, the vector's compressed bytes decoded as one
// stream (stream_vector: code-parallel, a lane per 4 bytes).  LENGTHS: per-vector decoded byte totals.
// MATERIALIZE: Arrow offsets and bytes at the first output byte of every vector computed from the totals.
template <int PASS, int KIND>
__global__ void __launch_bounds__(kStrMaxWarps * 32) k_stream_pass(const StrArgs a) {
	extern __shared__ __align__(128) uint8_t smem[];
	constexpr bool      kFsst = KIND == STR_FSST;
	__shared__ uint64_t fsym[kFsst ? 256 : 1];
	__shared__ uint8_t  flen[kFsst ? 256 : 1];
	const uint32_t      lane = threadIdx.x & 31u, warp = threadIdx.x >> 5, nwarps = blockDim.x >> 5;
	constexpr uint32_t  kPerWarp = str_per_warp(PASS, false);
	if constexpr (kFsst) {
		// code 255 (the escape) keeps an empty entry: stream_vector reads bytes past a stream's end as code 255
		for (uint32_t i = threadIdx.x; i < 256; i += blockDim.x) {
			fsym[i] = i == 255 ? 0ull : a.table->sym[i];
			flen[i] = i == 255 ? 0u : a.table->len[i];
		}
	}
	uint8_t*        wbase  = smem + warp * kPerWarp;
	PlanS*          plans  = reinterpret_cast<PlanS*>(wbase);
	uint8_t*        buf    = wbase + kStrPB * 64;
	const uint32_t* rows32 = reinterpret_cast<const uint32_t*>(buf);
	uint8_t*        win    = buf + kStrRows;
	__syncthreads();

	const uint64_t gw = static_cast<uint64_t>(blockIdx.x) * nwarps + warp;
	const uint64_t nw = static_cast<uint64_t>(gridDim.x) * nwarps;
	const uint64_t n  = a.col.n_vec;
	uint32_t       k  = 0;
	for (uint64_t v = gw; v < n; v += nw, ++k) {
		if (k % kStrPB == 0) {
			if (lane < kStrPB) {
				const uint64_t u = v + lane * nw;
				Plan           q {};
				if (u < n) { q = make_plan(a.col, static_cast<uint32_t>(u)); }
				plans[lane] = pack_plan(q, u < n);
			}
			__syncwarp();
		}
		const Plan p = unpack_plan(plans[k % kStrPB]);
		if (!p.ok) {
			if (lane == 0) {
				atomicOr(a.status, p.bw > p.ws ? STATUS_BAD_BW : STATUS_BAD_LAYOUT);
				if (PASS == STR_PASS_LENGTHS) { a.vec_total[v] = 0; }
			}
			continue;
		}
		if (lane == 0 && (k + 1) % kStrPB != 0) {
			// the next vector's packed row offsets towards L2
			const Plan q = unpack_plan(plans[(k + 1) % kStrPB]);
			const uintptr_t lo = (reinterpret_cast<uintptr_t>(q.src) + 15) & ~uintptr_t(15);
			const uintptr_t hi = (reinterpret_cast<uintptr_t>(q.src) + q.bytes) & ~uintptr_t(15);
			if (q.ok && hi > lo) { bulk_prefetch_l2(reinterpret_cast<const void*>(lo), static_cast<uint32_t>(hi - lo)); }
		}
		load_rows<false>(p, buf, lane, a.status);
		uint32_t       vn  = 0;
		const uint8_t* vb  = vector_bytes(a.col, static_cast<uint32_t>(v), &vn);
		bool           bad = false;
		StreamOut      o {};
		if (lane == 0 && v + nw < n) {
			// the warp's next vector's bytes towards L2 (the 16-byte aligned part inside them)
			uint32_t       nn = 0;
			const uint8_t* nb = vector_bytes(a.col, static_cast<uint32_t>(v + nw), &nn);
			const uintptr_t lo = (reinterpret_cast<uintptr_t>(nb) + 15) & ~uintptr_t(15);
			const uintptr_t hi = (reinterpret_cast<uintptr_t>(nb) + nn) & ~uintptr_t(15);
			if (hi > lo) { bulk_prefetch_l2(reinterpret_cast<const void*>(lo), static_cast<uint32_t>(hi - lo)); }
		}
		if constexpr (PASS == STR_PASS_LENGTHS) {
			const uint32_t tot = stream_vector<false, kFsst, kStrWindow>(rows32, vb, vn, fsym, flen, lane, o, &bad);
			if (lane == 0) {
				a.vec_total[v] = tot;
				if (bad) { atomicOr(a.status, STATUS_BAD_INDEX); }
			}
		} else {
			const uint64_t vbase = a.vec_base[v];
			const uint64_t vend  = a.vec_base[v + 1];
			if (vend < vbase || vend > a.bytes_cap) {
				if (lane == 0) { atomicOr(a.status, STATUS_BAD_LAYOUT); }
				__syncwarp();
				continue;
			}
			o.offsets          = a.offsets + v * kVec;
			o.bytes            = a.bytes;
			o.vbase            = vbase;
			o.win              = win;
			const uint32_t tot = stream_vector<true, kFsst, kStrWindow>(rows32, vb, vn, fsym, flen, lane, o, &bad);
			if (lane == 0) {
				if (v + 1 == n) { a.offsets[n * kVec] = static_cast<uint32_t>(vbase + tot); }
				if (bad || vbase + tot != vend) { atomicOr(a.status, STATUS_BAD_INDEX); }
			}
		}
		__syncwarp();
	}
}

// ---------------------------------------------------------------------------------------------------------
// Single-pass DICT decode (k_dict_pass): no lengths pass.  A vector's rows resolve to (dictionary start,
// length) through the packed row table; their lengths sum to the vector's total, which the warp publishes as
// soon as it has it; its first output byte is the sum of its column's earlier totals, read back from the
// earlier vectors' look-back words (a predecessor that has its inclusive prefix ends the walk).  Tickets hand
// out work in vector order, so every vector a warp waits for was taken by a warp that is already running and
// publishes without waiting on anything: the walk always ends.  Its spin is bounded all the same.
// ---------------------------------------------------------------------------------------------------------
constexpr uint64_t kLbAgg = 1ull << 62, kLbInc = 2ull << 62, kLbVal = (1ull << 62) - 1;
constexpr uint32_t kLookbackSpinLimit = 1u << 20;

__device__ __forceinline__ uint64_t ld_acquire_u64(const uint64_t* p) {
	uint64_t v;
	asm volatile("ld.acquire.gpu.global.u64 %0, [%1];" : "=l"(v) : "l"(p) : "memory");
	return v;
}
__device__ __forceinline__ void st_release_u64(uint64_t* p, uint64_t v) {
	asm volatile("st.release.gpu.global.u64 [%0], %1;" ::"l"(p), "l"(v) : "memory");
}

// Exclusive prefix of vector v's column (words: the column's look-back words, vector 0 first): walk back 32
// words at a time until a word with an inclusive prefix.  STATUS_TIMEOUT (and a partial sum) if a predecessor
// never publishes.
__device__ __forceinline__ uint64_t lookback(const uint64_t* words, uint32_t v, uint32_t lane, int* status) {
	uint64_t P     = 0;
	int64_t  j     = static_cast<int64_t>(v) - 1;
	uint32_t spins = 0;
	while (true) {
		const int64_t  idx  = j - static_cast<int64_t>(lane);
		const uint64_t f    = idx >= 0 ? ld_acquire_u64(words + idx) : kLbInc; // before vector 0: prefix 0
		const uint32_t inc  = __ballot_sync(0xFFFFFFFFu, (f >> 62) == 2u);
		const uint32_t emp  = __ballot_sync(0xFFFFFFFFu, (f >> 62) == 0u);
		const uint32_t upto = inc ? (((inc & (0u - inc)) << 1) - 1u) : 0xFFFFFFFFu; // lanes up to the nearest prefix
		if (emp & upto) {
			if (++spins > kLookbackSpinLimit) {
				if (lane == 0) { atomicOr(status, STATUS_TIMEOUT); }
				return P;
			}
			__nanosleep(64);
			continue;
		}
		P += warp_sum<uint64_t>(((upto >> lane) & 1u) ? (f & kLbVal) : 0ull);
		if (inc) { return P; }
		j -= 32;
	}
}

// Rows of one DICT vector into Arrow offsets and bytes from the first output byte vbase: 32 rows at a time (a
// row per lane, positions by a warp scan) into the warp's output window (put_row), which leaves in 16-byte
// stores.  tab: the packed row table (start | length << 24) of the dictionary's entry_c entries.  Returns the
// bytes written; *bad for codes outside the dictionary (such rows are empty).
template <bool R16>
__device__ __forceinline__ uint32_t dict_vector_out(const uint8_t* rows, const uint32_t* tab, uint32_t entry_c,
                                                    const uint8_t* dict, uint8_t* win, uint32_t* offs, uint8_t* bytes,
                                                    uint64_t vbase, uint32_t lane, bool* bad) {
	uint32_t* win32 = reinterpret_cast<uint32_t*>(win);
	uint64_t  W     = vbase & ~15ull; // output position of win[0]
	uint32_t  fill  = static_cast<uint32_t>(vbase & 15u);
	uint64_t  lo    = vbase; // first output byte the window may write
	if (lane == 0) { win32[fill >> 2] = 0; }
	__syncwarp();
	auto flush = [&](bool all) {
		const uint32_t full = fill & ~15u;
		const uint32_t upto = all ? fill : full;
		for (uint32_t c = 16 * lane; c < upto; c += 512) {
			const uint64_t g = W + c;
			if (g >= lo && c + 16 <= upto) {
				*reinterpret_cast<uint4*>(bytes + g) = *reinterpret_cast<const uint4*>(win + c);
			} else {
				for (uint32_t i = 0; i < 16 && c + i < upto; ++i) {
					if (g + i >= lo) { bytes[g + i] = win[c + i]; }
				}
			}
		}
		__syncwarp();
		if (!all) {
			if (lane == 0 && full != 0 && (fill & 15u) != 0) {
				*reinterpret_cast<uint4*>(win) = *reinterpret_cast<const uint4*>(win + full);
			}
			__syncwarp();
			W += full;
			fill &= 15u;
			lo = lo > W ? lo : W;
		}
	};
	auto ref = [&](uint32_t r, uint32_t* start, uint32_t* len) {
		const uint32_t code = row_at<R16>(rows, r);
		if (code >= entry_c) {
			*bad   = true;
			*start = 0;
			*len   = 0;
		} else {
			const uint32_t e = tab[code];
			*start           = e & 0xFFFFFFu;
			*len             = e >> 24;
		}
	};
	uint32_t vpos = 0, ns, nl;
	ref(lane, &ns, &nl);
	for (uint32_t b = 0; b < kVec / 32; ++b) {
		const uint32_t fs = ns, fl = nl;
		if (b + 1 < kVec / 32) { ref(32 * (b + 1) + lane, &ns, &nl); }
		const uint32_t inc = warp_inclusive_scan(fl, lane);
		const uint32_t o   = vpos + inc - fl;
		const uint32_t T   = __shfl_sync(0xFFFFFFFFu, inc, 31);
		offs[32 * b + lane] = static_cast<uint32_t>(vbase + o);
		if (fill + T > kStrWindow) { flush(false); }
		if (fill + T <= kStrWindow) {
			uint32_t   hk = 0, head = 0;
			const bool mid = put_row(win32, fill + (o - vpos), reinterpret_cast<const uint32_t*>(dict), fs, fl, &hk, &head);
			__syncwarp(); // every word's whole store lands before the rows that start inside it OR in
			if (mid) { atomicOr(win32 + hk, head); }
			fill += T;
		} else {
			// a batch larger than the window: straight to global memory after the window's pending bytes
			flush(true);
			uint8_t* dst = bytes + vbase + o;
			for (uint32_t i = 0; i < fl; ++i) { dst[i] = dict[fs + i]; }
			const uint64_t pos = vbase + vpos + T;
			W                  = pos & ~15ull;
			fill               = static_cast<uint32_t>(pos & 15u);
			lo                 = pos;
			__syncwarp();
			if (lane == 0) { win32[fill >> 2] = 0; }
		}
		vpos += T;
		__syncwarp();
	}
	flush(true);
	return vpos;
}

template <bool R16, bool SMDICT>
__global__ void __launch_bounds__(kStrMaxWarps * 32) k_dict_pass(const StrSetArgs s) {
	extern __shared__ __align__(128) uint8_t smem[];
	__shared__ uint32_t s_chunk;
	const uint32_t      lane = threadIdx.x & 31u, warp = threadIdx.x >> 5, nwarps = blockDim.x >> 5;
	constexpr uint32_t  kPerWarp = str_rows_bytes(R16) + kStrWindow;
	uint8_t*            rows     = smem + warp * kPerWarp;
	uint8_t*            win      = rows + str_rows_bytes(R16);
	uint8_t*            sdict    = smem + nwarps * kPerWarp;
	uint32_t*           stab     = reinterpret_cast<uint32_t*>(sdict + s.dict_cap);
	int64_t             loaded   = -1;
	for (;;) {
		if (threadIdx.x == 0) {
			s_chunk = static_cast<uint32_t>(atomicAdd(reinterpret_cast<unsigned long long*>(s.flags), 1ull));
		}
		__syncthreads();
		const uint32_t ch = s_chunk;
		if (ch >= s.n_chunks) { break; }
		const uint32_t col = s.chunk_col ? __ldg(s.chunk_col + ch) : 0u;
		const StrArgs& A   = s.cols[col];
		if constexpr (SMDICT) {
			if (static_cast<int64_t>(col) != loaded) {
				// the column's decoded dictionary (cudaMalloc'd, 16 bytes of slack) and row table
				const uint32_t nb16 = static_cast<uint32_t>((A.dict_bytes_n + 15) / 16);
				const uint4*   src  = reinterpret_cast<const uint4*>(A.dict_bytes);
				for (uint32_t i = threadIdx.x; i < nb16; i += blockDim.x) { reinterpret_cast<uint4*>(sdict)[i] = __ldg(src + i); }
				for (uint32_t i = threadIdx.x; i < A.entry_c; i += blockDim.x) { stab[i] = __ldg(A.dict_rows + i); }
				loaded = col;
			}
		}
		__syncthreads(); // also: every thread has read s_chunk before thread 0 overwrites it
		const uint32_t v0    = s.chunk_v0 ? __ldg(s.chunk_v0 + ch) : ch * s.chunk_w;
		const uint32_t n_vec = A.col.n_vec;
		const uint32_t v     = v0 + warp;
		if (warp >= s.chunk_w || v >= n_vec || v >= v0 + s.chunk_w) { continue; }
		const uint8_t*  dict    = SMDICT ? sdict : A.dict_bytes;
		const uint32_t* tab     = SMDICT ? stab : A.dict_rows;
		const uint32_t  entry_c = A.entry_c;
		uint64_t*       words   = s.flags + 1 + A.item_base;
		const Plan      p       = make_plan(A.col, v);
		bool            bad     = false;
		bool            ok      = p.ok;
		if (!ok && lane == 0) { atomicOr(s.status, p.bw > p.ws ? STATUS_BAD_BW : STATUS_BAD_LAYOUT); }
		if (ok) { ok = load_rows<R16>(p, rows, lane, s.status); }
		// the vector's total: every row's length
		uint32_t T = 0;
		if (ok) {
			uint32_t sum = 0;
			for (uint32_t b = 0; b < kVec / 32; ++b) {
				const uint32_t code = row_at<R16>(rows, 32 * b + lane);
				if (code < entry_c) {
					sum += tab[code] >> 24;
				} else {
					bad = true;
				}
			}
			T = warp_sum(sum);
		}
		// every vector publishes (also one that failed: its successors wait for it)
		if (lane == 0) { st_release_u64(words + v, (v == 0 ? kLbInc : kLbAgg) | T); }
		const uint64_t P = v == 0 ? 0ull : lookback(words, v, lane, s.status);
		if (lane == 0 && v > 0) { st_release_u64(words + v, kLbInc | (P + T)); }
		uint32_t*      offsets = s.out_offsets ? s.out_offsets : A.offsets;
		uint8_t*       bytes   = s.out_offsets ? s.out_bytes : A.bytes;
		const uint64_t cap     = s.out_offsets ? s.out_cap : A.bytes_cap;
		uint32_t*      offs    = offsets + static_cast<uint64_t>(v) * kVec;
		if (P + T > cap || P + T >= (1ull << 32)) {
			if (lane == 0) { atomicOr(s.status, STATUS_BAD_LAYOUT); }
		} else if (!ok) {
			for (uint32_t r = lane; r < kVec; r += 32) { offs[r] = static_cast<uint32_t>(P); }
		} else {
			const uint32_t got = dict_vector_out<R16>(rows, tab, entry_c, dict, win, offs, bytes, P, lane, &bad);
			if (got != T) { bad = true; }
		}
		if (lane == 0 && v + 1 == n_vec) { offsets[static_cast<uint64_t>(n_vec) * kVec] = static_cast<uint32_t>(P + T); }
		if (__any_sync(0xFFFFFFFFu, bad) && lane == 0) { atomicOr(s.status, STATUS_BAD_INDEX); }
		__syncwarp();
	}
}

// Single-pass FSST / BYTE_ARR decode (no lengths pass, no scan).  A warp takes vectors by ticket (lb[0]), in
// vector order, so every vector it waits for was taken by a running warp that publishes without waiting.  Per
// vector: its rows; its decoded total -- the sum of its codes' symbol lengths when no escape is among its bytes,
// else the escape-aware walk of stream_vector (a BYTE_ARR vector's total is its compressed length) -- published
// in its look-back word lb[1 + v]; its first output byte from the earlier vectors' words (lookback); then its
// offsets and bytes (stream_vector), whose total must match.
template <int KIND>
__global__ void __launch_bounds__(kStrMaxWarps * 32) k_stream_single(const StrArgs a, uint64_t* lb) {
	extern __shared__ __align__(128) uint8_t smem[];
	constexpr bool      kFsst = KIND == STR_FSST;
	__shared__ uint64_t fsym[kFsst ? 256 : 1];
	__shared__ uint8_t  flen[kFsst ? 256 : 1];
	const uint32_t      lane = threadIdx.x & 31u, warp = threadIdx.x >> 5;
	if constexpr (kFsst) {
		// code 255 (the escape) keeps an empty entry: stream_vector reads bytes past a stream's end as code 255
		for (uint32_t i = threadIdx.x; i < 256; i += blockDim.x) {
			fsym[i] = i == 255 ? 0ull : a.table->sym[i];
			flen[i] = i == 255 ? 0u : a.table->len[i];
		}
	}
	uint8_t*        buf    = smem + warp * kStreamSinglePerWarp;
	const uint32_t* rows32 = reinterpret_cast<const uint32_t*>(buf);
	uint8_t*        win    = buf + kStrRows;
	__syncthreads();
	const uint64_t n     = a.col.n_vec;
	uint64_t*      words = lb + 1;
	for (;;) {
		unsigned long long t = 0;
		if (lane == 0) { t = atomicAdd(reinterpret_cast<unsigned long long*>(lb), 1ull); }
		const uint64_t v = __shfl_sync(0xFFFFFFFFu, t, 0);
		if (v >= n) { break; }
		const Plan     p  = make_plan(a.col, static_cast<uint32_t>(v));
		uint32_t       vn = 0;
		const uint8_t* vb = vector_bytes(a.col, static_cast<uint32_t>(v), &vn);
		if (lane == 0) {
			// the vector's bytes towards L2 while its rows decode (the 16-byte aligned part inside them)
			const uintptr_t lo = (reinterpret_cast<uintptr_t>(vb) + 15) & ~uintptr_t(15);
			const uintptr_t hi = (reinterpret_cast<uintptr_t>(vb) + vn) & ~uintptr_t(15);
			if (hi > lo) { bulk_prefetch_l2(reinterpret_cast<const void*>(lo), static_cast<uint32_t>(hi - lo)); }
		}
		const bool ok  = p.ok;
		bool       bad = false;
		if (!ok && lane == 0) { atomicOr(a.status, p.bw > p.ws ? STATUS_BAD_BW : STATUS_BAD_LAYOUT); }
		uint32_t T = 0;
		if (ok) {
			load_rows<false>(p, buf, lane, a.status);
			const uint32_t L = stream_rows_length(rows32, vn, lane, &bad);
			T                = L;
			if (kFsst && !fsst_plain_total(vb, L, flen, lane, &T)) {
				StreamOut o {};
				T = stream_vector<false, true, kStrWindow>(rows32, vb, vn, fsym, flen, lane, o, &bad);
			}
		}
		// every vector publishes (also one that failed: its successors wait for it)
		if (lane == 0) { st_release_u64(words + v, (v == 0 ? kLbInc : kLbAgg) | T); }
		const uint64_t P = v == 0 ? 0ull : lookback(words, static_cast<uint32_t>(v), lane, a.status);
		if (lane == 0 && v > 0) { st_release_u64(words + v, kLbInc | (P + T)); }
		uint32_t* offs = a.offsets + v * kVec;
		if (P + T > a.bytes_cap || P + T >= (1ull << 32)) {
			if (lane == 0) { atomicOr(a.status, STATUS_BAD_LAYOUT); }
		} else if (!ok) {
			for (uint32_t r = lane; r < kVec; r += 32) { offs[r] = static_cast<uint32_t>(P); }
		} else {
			StreamOut o {offs, a.bytes, P, win};
			const uint32_t got = stream_vector<true, kFsst, kStrWindow>(rows32, vb, vn, fsym, flen, lane, o, &bad);
			if (got != T) { bad = true; }
		}
		if (lane == 0 && v + 1 == n) { a.offsets[n * kVec] = static_cast<uint32_t>(P + T); }
		if (__any_sync(0xFFFFFFFFu, bad) && lane == 0) { atomicOr(a.status, STATUS_BAD_INDEX); }
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

// ---------------------------------------------------------------------------------------------------------
// Host launchers
// ---------------------------------------------------------------------------------------------------------
uint32_t str_smem_per_warp(bool rows16) { return str_per_warp(STR_PASS_MATERIALIZE, rows16); }

cudaError_t launch_fsst_dict(const uint8_t* lens, const uint8_t* comp, uint64_t comp_size, uint32_t entry_c,
                             const FsstTable* tab, uint32_t* ends, uint8_t* bytes, uint64_t cap, int* status,
                             cudaStream_t s) {
	if (entry_c == 0) { return cudaSuccess; }
	k_fsst_dict<<<1, 1024, 0, s>>>(lens, comp, comp_size, entry_c, tab, ends, bytes, cap, status);
	++launch_counter();
	return cudaGetLastError();
}

// Launch one pass of kernel fn over the column's vectors with `warps` warps per CTA and as many CTAs per SM as
// shared memory allows (no more CTAs than there are vectors for their warps).  *set / *mu: the kernel's dynamic
// shared-memory limit set so far and its lock.  sm_count 0: the SM count of the library's per-device state.
template <class F>
static cudaError_t launch_pass(F fn, uint32_t* set, std::mutex* mu, const StrArgs& a, int warps, uint32_t dyn_smem,
                               cudaStream_t s, int sm_count) {
	{
		std::lock_guard<std::mutex> lk(*mu);
		if (dyn_smem > *set) {
			const cudaError_t e = cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, dyn_smem);
			if (e != cudaSuccess) { return e; }
			*set = dyn_smem;
		}
	}
	if (sm_count <= 0) {
		const Device* dev = current_device();
		if (!dev) { return cudaErrorUnknown; }
		sm_count = dev->sm_count;
	}
	int         per_sm = 0;
	cudaError_t e      = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, fn, warps * 32, dyn_smem);
	if (e != cudaSuccess) { return e; }
	if (per_sm < 1) { return cudaErrorInvalidConfiguration; }
	const uint64_t need = (a.col.n_vec + warps - 1) / warps;
	uint64_t       grid = static_cast<uint64_t>(sm_count) * per_sm;
	grid                = grid < need ? grid : need;
	if (grid == 0) { return cudaSuccess; }
	fn<<<static_cast<unsigned>(grid), warps * 32, dyn_smem, s>>>(a);
	++launch_counter();
	return cudaGetLastError();
}

template <int PASS, int KIND, int SM, bool R16 = false>
static cudaError_t launch_str_kernel(const StrArgs& a, int warps, uint32_t dyn_smem, cudaStream_t s, int sm_count) {
	static std::mutex mu;
	static uint32_t   set = 0;
	return launch_pass(k_str_pass<PASS, KIND, SM, R16>, &set, &mu, a, warps, dyn_smem, s, sm_count);
}

template <int PASS, int KIND>
static cudaError_t launch_stream_kernel(const StrArgs& a, int warps, uint32_t dyn_smem, cudaStream_t s, int sm_count) {
	static std::mutex mu;
	static uint32_t   set = 0;
	return launch_pass(k_stream_pass<PASS, KIND>, &set, &mu, a, warps, dyn_smem, s, sm_count);
}

cudaError_t launch_str_lengths(const StrArgs& a, int sm_count, cudaStream_t s) {
	constexpr int      w  = kStrLenWarps;
	const uint32_t     sm = w * str_per_warp(STR_PASS_LENGTHS, a.rows16);
	switch (a.kind) {
	case STR_DICT:
		if (a.rows16) {
			return a.ends_in_smem ? launch_str_kernel<STR_PASS_LENGTHS, STR_DICT, SM_ENDS, true>(a, w, sm + str_ends_smem(a), s, sm_count)
			                      : launch_str_kernel<STR_PASS_LENGTHS, STR_DICT, SM_NONE, true>(a, w, sm, s, sm_count);
		}
		return a.ends_in_smem ? launch_str_kernel<STR_PASS_LENGTHS, STR_DICT, SM_ENDS>(a, w, sm + str_ends_smem(a), s, sm_count)
		                      : launch_str_kernel<STR_PASS_LENGTHS, STR_DICT, SM_NONE>(a, w, sm, s, sm_count);
	case STR_FSST: return launch_stream_kernel<STR_PASS_LENGTHS, STR_FSST>(a, w, sm, s, sm_count);
	case STR_FSST12: return launch_str_kernel<STR_PASS_LENGTHS, STR_FSST12, SM_NONE>(a, w, sm, s, sm_count);
	default: return launch_stream_kernel<STR_PASS_LENGTHS, STR_BYTES>(a, w, sm, s, sm_count);
	}
}

uint32_t dict_pass_smem_per_warp(bool rows16) { return str_rows_bytes(rows16) + kStrWindow; }

template <bool R16, bool SMDICT>
static cudaError_t launch_dict_pass_t(const StrSetArgs& a, int warps, uint32_t dyn_smem, cudaStream_t s, int sm_count) {
	auto* const       fn = k_dict_pass<R16, SMDICT>;
	static std::mutex mu;
	static uint32_t   set = 0;
	{
		std::lock_guard<std::mutex> lk(mu);
		if (dyn_smem > set) {
			const cudaError_t e = cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, dyn_smem);
			if (e != cudaSuccess) { return e; }
			set = dyn_smem;
		}
	}
	if (sm_count <= 0) {
		const Device* dev = current_device();
		if (!dev) { return cudaErrorUnknown; }
		sm_count = dev->sm_count;
	}
	int         per_sm = 0;
	cudaError_t e      = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, fn, warps * 32, dyn_smem);
	if (e != cudaSuccess) { return e; }
	if (per_sm < 1) { return cudaErrorInvalidConfiguration; }
	uint64_t grid = static_cast<uint64_t>(sm_count) * per_sm;
	grid          = grid < a.n_chunks ? grid : a.n_chunks;
	if (grid == 0) { return cudaSuccess; }
	fn<<<static_cast<unsigned>(grid), warps * 32, dyn_smem, s>>>(a);
	++launch_counter();
	return cudaGetLastError();
}

cudaError_t launch_dict_pass(const StrSetArgs& a, bool rows16, int warps, uint32_t dyn_smem, cudaStream_t s,
                             int sm_count) {
	if (warps < 1 || warps > kStrMaxWarps || a.chunk_w != static_cast<uint32_t>(warps)) {
		return cudaErrorInvalidValue;
	}
	const bool sm = a.dict_cap != 0;
	if (rows16) {
		return sm ? launch_dict_pass_t<true, true>(a, warps, dyn_smem, s, sm_count)
		          : launch_dict_pass_t<true, false>(a, warps, dyn_smem, s, sm_count);
	}
	return sm ? launch_dict_pass_t<false, true>(a, warps, dyn_smem, s, sm_count)
	          : launch_dict_pass_t<false, false>(a, warps, dyn_smem, s, sm_count);
}

template <int KIND>
static cudaError_t launch_stream_single_t(const StrArgs& a, uint64_t* lb, cudaStream_t s, int sm_count) {
	auto* const        fn    = k_stream_single<KIND>;
	constexpr int      warps = kStrMaxWarps;
	constexpr uint32_t smem  = warps * kStreamSinglePerWarp;
	static std::mutex  mu;
	static bool        set = false;
	{
		std::lock_guard<std::mutex> lk(mu);
		if (!set) {
			const cudaError_t e = cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, smem);
			if (e != cudaSuccess) { return e; }
			set = true;
		}
	}
	if (sm_count <= 0) {
		const Device* dev = current_device();
		if (!dev) { return cudaErrorUnknown; }
		sm_count = dev->sm_count;
	}
	// one CTA per SM (its 32 warps take vectors by ticket); no more warps than vectors
	const uint64_t need = (static_cast<uint64_t>(a.col.n_vec) + warps - 1) / warps;
	const uint64_t grid = need < static_cast<uint64_t>(sm_count) ? need : static_cast<uint64_t>(sm_count);
	if (grid == 0) { return cudaSuccess; }
	fn<<<static_cast<unsigned>(grid), warps * 32, smem, s>>>(a, lb);
	++launch_counter();
	return cudaGetLastError();
}

cudaError_t launch_stream_single(const StrArgs& a, uint64_t* lb, cudaStream_t s, int sm_count) {
	switch (a.kind) {
	case STR_FSST: return launch_stream_single_t<STR_FSST>(a, lb, s, sm_count);
	case STR_BYTES: return launch_stream_single_t<STR_BYTES>(a, lb, s, sm_count);
	default: return cudaErrorInvalidValue;
	}
}

cudaError_t launch_scan_totals(const uint64_t* total, uint64_t* base, uint64_t n, cudaStream_t s) {
	k_scan_totals<<<1, 1024, 0, s>>>(total, base, n);
	++launch_counter();
	return cudaGetLastError();
}

cudaError_t launch_str_materialize(const StrArgs& a, int warps, uint32_t dyn_smem, cudaStream_t s, int sm_count) {
	switch (a.kind) {
	case STR_DICT:
		if (a.rows16) {
			return a.dict_in_smem ? launch_str_kernel<STR_PASS_MATERIALIZE, STR_DICT, SM_BYTES, true>(a, warps, dyn_smem, s, sm_count)
			                      : launch_str_kernel<STR_PASS_MATERIALIZE, STR_DICT, SM_NONE, true>(a, warps, dyn_smem, s, sm_count);
		}
		return a.dict_in_smem ? launch_str_kernel<STR_PASS_MATERIALIZE, STR_DICT, SM_BYTES>(a, warps, dyn_smem, s, sm_count)
		                      : launch_str_kernel<STR_PASS_MATERIALIZE, STR_DICT, SM_NONE>(a, warps, dyn_smem, s, sm_count);
	case STR_FSST: return launch_stream_kernel<STR_PASS_MATERIALIZE, STR_FSST>(a, warps, dyn_smem, s, sm_count);
	case STR_FSST12: return launch_str_kernel<STR_PASS_MATERIALIZE, STR_FSST12, SM_NONE>(a, warps, dyn_smem, s, sm_count);
	default: return launch_stream_kernel<STR_PASS_MATERIALIZE, STR_BYTES>(a, warps, dyn_smem, s, sm_count);
	}
}

} // namespace flsgpu

// =========================================================================================================
// Allocation-free decode of FSST / BYTE_ARR string pages (fls_gpu_decode_fsst_page_noalloc).
//
// The string plan keeps its scratch (per-vector byte totals and first-byte bases, the FSST table) in
// cudaMalloc'd buffers and reports device errors through the library's per-device status word, which is
// cudaMalloc'd on a device's first use.  This variant keeps the same scratch in one array compiled into the
// library and reports errors through the caller's status word, so nothing on its path allocates: it reads the
// SM count itself instead of going through current_device().  In exchange a page may hold at most
// kNoAllocMaxVectors vectors.
// =========================================================================================================
namespace flsgpu {

constexpr uint32_t kNoAllocMaxVectors = 8192; // 8,388,608 rows per call

struct NoAllocLayout {
	static constexpr size_t kTable = 0;                                        // FsstTable (2304 B)
	static constexpr size_t kTotal = kTable + ((sizeof(FsstTable) + 255) & ~size_t(255));
	static constexpr size_t kBase  = kTotal + 8 * (kNoAllocMaxVectors + 1);
	static constexpr size_t kBytes = kBase + 8 * (kNoAllocMaxVectors + 1);
};
static_assert(NoAllocLayout::kBytes == FLS_NOALLOC_SCRATCH_BYTES, "the header states the scratch size");
static_assert(kNoAllocMaxVectors == FLS_NOALLOC_MAX_VECTORS, "the header states the vector limit");

// Every GPU that loads the library holds this array until the process exits.
static __device__ __align__(256) uint8_t g_noalloc_scratch[NoAllocLayout::kBytes];

// Device address of g_noalloc_scratch on the current device, looked up once per device on the first call
// (host code cannot use the symbol itself: on the host it names a stand-in, not device memory).
static uint8_t* noalloc_scratch(int dev) {
	static uint8_t*   addr[64] = {};
	static std::mutex mu;
	if (dev < 0 || dev >= 64) { return nullptr; }
	std::lock_guard<std::mutex> lk(mu);
	if (!addr[dev]) {
		void* p = nullptr;
		if (cudaGetSymbolAddress(&p, g_noalloc_scratch) != cudaSuccess || p == nullptr) { return nullptr; }
		addr[dev] = static_cast<uint8_t*>(p);
	}
	return addr[dev];
}

int fsst_import_table(const uint8_t* buf, uint64_t avail, FsstTable* t, uint64_t* used);

// n bytes from device memory into host memory in the stream's order (after the work queued on it before).
static bool read_in_stream_order(void* dst, const void* src, uint64_t n, cudaStream_t s) {
	return cudaMemcpyAsync(dst, src, n, cudaMemcpyDeviceToHost, s) == cudaSuccess &&
	       cudaStreamSynchronize(s) == cudaSuccess;
}

} // namespace flsgpu

extern "C" int fls_gpu_decode_fsst_page_noalloc(const uint8_t* d_page, uint64_t page_size, const uint8_t* d_dict,
                                                uint64_t dict_size, uint32_t* d_offsets, uint8_t* d_bytes,
                                                uint64_t bytes_cap, int* d_status, void* stream) {
	using namespace flsgpu;
	if (!d_page || !d_offsets || !d_status || (!d_bytes && bytes_cap) ||
	    (reinterpret_cast<uintptr_t>(d_bytes) & 15u) != 0 || bytes_cap >= (1ull << 32)) {
		return FLS_ERR_ARG;
	}
	cudaStream_t   s = static_cast<cudaStream_t>(stream);
	uint8_t        hdr[8 + 4 * 5];
	const uint64_t take = page_size < sizeof(hdr) ? page_size : sizeof(hdr);
	if (take < 8) { return FLS_ERR_FORMAT; }
	// the page may have been written by work the caller queued on this stream: read it in the stream's order
	if (!read_in_stream_order(hdr, d_page, take, s)) { return FLS_ERR_CUDA; }
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
	int dev = 0, sms = 0;
	if (cudaGetDevice(&dev) != cudaSuccess ||
	    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess || sms <= 0) {
		return FLS_ERR_CUDA;
	}
	uint8_t* scratch = noalloc_scratch(dev);
	if (!scratch) { return FLS_ERR_CUDA; }
	FsstTable tab {};
	if (kind == STR_FSST) {
		// dict_hdr_t followed by the exported symbol table (at most FSST_MAXHEADER = 2066 bytes)
		uint8_t        h[8 + 2066];
		const uint64_t n = dict_size < sizeof(h) ? dict_size : sizeof(h);
		if (!d_dict || n < 8 + 17) { return FLS_ERR_FORMAT; }
		if (!read_in_stream_order(h, d_dict, n, s)) { return FLS_ERR_CUDA; }
		const int rc = fsst_import_table(h + 8, n - 8, &tab, nullptr);
		if (rc != FLS_OK) { return rc; }
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
	// the table is the only scratch content a call relies on; totals and bases are rewritten in full by every
	// call.  A copy from pageable host memory has read its source when cudaMemcpyAsync returns, so the table may
	// live in this stack frame.
	if (kind == STR_FSST &&
	    cudaMemcpyAsync(scratch + NoAllocLayout::kTable, &tab, sizeof(tab), cudaMemcpyHostToDevice, s) != cudaSuccess) {
		return FLS_ERR_CUDA;
	}
	StrArgs a {};
	a.col       = c;
	a.kind      = kind;
	a.table     = reinterpret_cast<const FsstTable*>(scratch + NoAllocLayout::kTable);
	a.vec_total = reinterpret_cast<uint64_t*>(scratch + NoAllocLayout::kTotal);
	a.vec_base  = reinterpret_cast<const uint64_t*>(scratch + NoAllocLayout::kBase);
	a.offsets   = d_offsets;
	a.bytes     = d_bytes;
	a.bytes_cap = bytes_cap;
	a.status    = d_status;
	if (launch_str_lengths(a, sms, s) != cudaSuccess ||
	    launch_scan_totals(a.vec_total, reinterpret_cast<uint64_t*>(scratch + NoAllocLayout::kBase), vec_c, s) !=
	        cudaSuccess ||
	    launch_str_materialize(a, kStrLenWarps, kStrLenWarps * str_smem_per_warp(false), s, sms) != cudaSuccess) {
		return FLS_ERR_CUDA;
	}
	return FLS_OK;
}
