// Expression selection on the B200 (include/fls_select.h): the exact-size wizard, the per-vector statistics of
// the learned selector, and the MLP kernels (forward, gradient, Adam, graph-replayed training).
//
// Per-vector work runs warp per vector with every thread holding 32 contiguous values in registers: thread t
// holds original positions R(t) = (t % 16) * 64 + 32 * (t / 16) .. + 31.  In the unified transposed layout
// that run is exactly
//   * W = 32: the whole lane t;
//   * W = 64: half of lane t % 16, the other half in thread t ^ 16;
//   * W = 16 (the RLE run index): two whole lanes, [0,16) and [16,32) of the run.
// and the rsum / unrsum chains visit a lane in ascending original order, so FFOR, DELTA and RLE sizes come out
// of one read of the values.
#include "fls_device.cuh"
#include "fls_runtime.h"
#include "fls_b200.h"
#include "fls_select.h"
#include "fls_strings.cuh"
#include "fls_strplan.h"

#include <algorithm>
#include <cmath>
#include <cstring>
#include <map>
#include <memory>
#include <random>
#include <vector>

namespace flsgpu {
namespace sel {

constexpr int      K        = FLS_SEL_K;
constexpr int      NF       = FLS_SEL_FEATURES;
constexpr int      H        = FLS_SEL_HIDDEN;
constexpr uint64_t kEmpty   = ~0ull;      // empty key of the hash tables; the value ~0 itself has a slot of its own
constexpr uint32_t kNoPos   = 0xFFFFFFFFu;
constexpr uint32_t kMaxVecPerChunk = 64;
constexpr int      kWarps   = 8;

struct Col {
	const uint8_t* values;
	uint64_t       n_vec;
	uint32_t       width;
	uint32_t       sgn;
};

// A work item: vector `vec` of column `col`; `chunk` its chunk, `cpos` its index inside the chunk.
struct Item {
	uint32_t col;
	uint32_t chunk;
	uint32_t vec;
	uint32_t cpos;
};

template <int W>
struct UT;
template <>
struct UT<32> {
	using T = uint32_t;
};
template <>
struct UT<64> {
	using T = uint64_t;
};

__device__ __forceinline__ uint32_t bits_of(uint64_t d) { return d ? 64u - static_cast<uint32_t>(__clzll(d)) : 0u; }

template <class T>
__device__ __forceinline__ T warp_min(T x) {
#pragma unroll
	for (int d = 16; d > 0; d >>= 1) {
		const T y = __shfl_xor_sync(0xFFFFFFFFu, x, d);
		x         = y < x ? y : x;
	}
	return x;
}
template <class T>
__device__ __forceinline__ T warp_max(T x) {
#pragma unroll
	for (int d = 16; d > 0; d >>= 1) {
		const T y = __shfl_xor_sync(0xFFFFFFFFu, x, d);
		x         = y > x ? y : x;
	}
	return x;
}

__device__ __forceinline__ uint32_t thread_run(uint32_t t) { return (t % 16) * 64 + 32 * (t / 16); }
// Lane whose run holds original position R(t) - 1 (t > 0).
__device__ __forceinline__ uint32_t prev_run_lane(uint32_t t) { return t >= 16 ? t - 16 : t + 15; }
// Thread runs in original order: virtual position u = 2 (t % 16) + t / 16.
__device__ __forceinline__ uint32_t lane_of_virtual(uint32_t u) { return (u >> 1) + 16 * (u & 1); }
__device__ __forceinline__ uint32_t virtual_of_lane(uint32_t t) { return 2 * (t % 16) + t / 16; }

// Exclusive sum of c over the thread runs in original order.
__device__ __forceinline__ uint32_t run_exclusive(uint32_t c, uint32_t lane) {
	const uint32_t cv  = __shfl_sync(0xFFFFFFFFu, c, lane_of_virtual(lane));
	const uint32_t inc = warp_inclusive_scan(cv, lane);
	return __shfl_sync(0xFFFFFFFFu, inc - cv, virtual_of_lane(lane));
}

template <int W>
__device__ __forceinline__ void load_run(const Col& c, uint64_t v, uint32_t lane, typename UT<W>::T (&x)[32]) {
	using T          = typename UT<W>::T;
	const uint4* src = reinterpret_cast<const uint4*>(c.values + (v * 1024 + thread_run(lane)) * sizeof(T));
	constexpr int n  = 32 * sizeof(T) / 16;
	uint4         b[n];
#pragma unroll
	for (int i = 0; i < n; ++i) { b[i] = __ldg(src + i); }
#pragma unroll
	for (int i = 0; i < n; ++i) {
		if constexpr (W == 32) {
			x[4 * i] = b[i].x, x[4 * i + 1] = b[i].y, x[4 * i + 2] = b[i].z, x[4 * i + 3] = b[i].w;
		} else {
			x[2 * i]     = (static_cast<uint64_t>(b[i].y) << 32) | b[i].x;
			x[2 * i + 1] = (static_cast<uint64_t>(b[i].w) << 32) | b[i].z;
		}
	}
}

// The size-model quantities of one vector (warp-uniform results).
struct Parts {
	uint32_t bw_f, bw_d, bw_i, runs;
	uint32_t start_mask; // this thread's run starts (bit i: original position R(t) + i starts a run)
};

template <int W>
__device__ __forceinline__ Parts vector_parts(const typename UT<W>::T (&x)[32], uint32_t lane, bool sgn) {
	using T      = typename UT<W>::T;
	const T flip = sgn ? (T(1) << (W - 1)) : T(0);
	Parts   P;
	// FFOR: range of the values (signed order through the flipped top bit)
	T mn = x[0] ^ flip, mx = mn;
#pragma unroll
	for (int i = 1; i < 32; ++i) {
		const T k = x[i] ^ flip;
		mn        = k < mn ? k : mn;
		mx        = k > mx ? k : mx;
	}
	mn     = warp_min(mn);
	mx     = warp_max(mx);
	P.bw_f = bits_of(static_cast<uint64_t>(static_cast<T>(mx - mn)));
	// DELTA: the unrsum chains of the transposed layout visit a lane's values in ascending original order, so
	// a chain is a run of contiguous original positions (W = 32: this thread's 32; W = 64: 64, this thread's
	// and its partner's); every chain's first difference is 0
	T dmn = flip, dmx = flip;
#pragma unroll
	for (int c = 1; c < 32; ++c) {
		const T k = static_cast<T>(x[c] - x[c - 1]) ^ flip;
		dmn       = k < dmn ? k : dmn;
		dmx       = k > dmx ? k : dmx;
	}
	if constexpr (W == 64) {
		const T lower = __shfl_xor_sync(0xFFFFFFFFu, x[31], 16);
		if (lane >> 4) {
			const T k = static_cast<T>(x[0] - lower) ^ flip;
			dmn       = k < dmn ? k : dmn;
			dmx       = k > dmx ? k : dmx;
		}
	}
	dmn    = warp_min(dmn);
	dmx    = warp_max(dmx);
	P.bw_d = bits_of(static_cast<uint64_t>(static_cast<T>(dmx - dmn)));
	// RLE: run starts in original order
	const T  prev = __shfl_sync(0xFFFFFFFFu, x[31], prev_run_lane(lane));
	uint32_t sm   = (lane == 0 || x[0] != prev) ? 1u : 0u;
#pragma unroll
	for (int i = 1; i < 32; ++i) { sm |= (x[i] != x[i - 1] ? 1u : 0u) << i; }
	P.start_mask = sm;
	P.runs       = warp_sum(static_cast<uint32_t>(__popc(sm)));
	// the u16 run index: each of its chains is 16 contiguous positions (this thread's [0,16) and [16,32)), so
	// its deltas are the run starts inside a chain (0 or 1) and the range is 1 as soon as one run starts there
	P.bw_i = __any_sync(0xFFFFFFFFu, (sm & 0xFFFEFFFEu) != 0) ? 1u : 0u;
	return P;
}

__device__ __forceinline__ uint32_t pack_parts(const Parts& p) {
	return p.bw_f | (p.bw_d << 7) | (p.bw_i << 14) | (p.runs << 19);
}

// ---------------------------------------------------------------------------------------------------------
// Statistics of the learned selector (one warp, one vector).  hkeys / hcnt: this warp's 2048-slot table.
// ---------------------------------------------------------------------------------------------------------
constexpr uint32_t kHSlots = 2048;

__device__ __forceinline__ uint32_t hash_slot(uint64_t x, uint32_t bits) {
	return static_cast<uint32_t>((x * 0x9E3779B97F4A7C15ull) >> (64 - bits));
}

template <int W>
__device__ void vector_features(const typename UT<W>::T (&x)[32], uint32_t lane, bool sgn, const Parts& P,
                                uint64_t* hkeys, uint32_t* hcnt, float* out) {
	using T             = typename UT<W>::T;
	const T        flip = sgn ? (T(1) << (W - 1)) : T(0);
	const uint32_t sm   = P.start_mask;
	// distinct values and the top multiplicity (exact: 1024 values in 2048 slots; the key ~0 counts aside)
	uint32_t sentinel = 0;
#pragma unroll
	for (int i = 0; i < 32; ++i) {
		const uint64_t key = static_cast<uint64_t>(x[i]);
		if (key == kEmpty) {
			++sentinel;
			continue;
		}
		uint32_t h = hash_slot(key, 11);
		for (uint32_t probe = 0; probe < kHSlots; ++probe) {
			const uint64_t old = atomicCAS(reinterpret_cast<unsigned long long*>(hkeys + h), kEmpty, key);
			if (old == kEmpty || old == key) {
				atomicAdd(hcnt + h, 1u);
				break;
			}
			h = (h + 1) & (kHSlots - 1);
		}
	}
	__syncwarp();
	uint32_t dv = 0, top = 0;
	for (uint32_t s = lane; s < kHSlots; s += 32) {
		const uint32_t c = hcnt[s];
		dv += c ? 1u : 0u;
		top = c > top ? c : top;
		hkeys[s] = kEmpty;
		hcnt[s]  = 0;
	}
	dv       = warp_sum(dv);
	top      = warp_max(top);
	sentinel = warp_sum(sentinel);
	if (sentinel) {
		++dv;
		top = sentinel > top ? sentinel : top;
	}
	// adjacency in original order: increases, decreases, largest |difference|
	const T  prev = __shfl_sync(0xFFFFFFFFu, x[31], prev_run_lane(lane));
	uint32_t inc = 0, dec = 0, bw_a = 0;
#pragma unroll
	for (int i = 0; i < 32; ++i) {
		if (i == 0 && lane == 0) { continue; }
		const T a = (i == 0 ? prev : x[i - 1]);
		const T b = x[i];
		inc += ((b ^ flip) > (a ^ flip)) ? 1u : 0u;
		dec += ((b ^ flip) < (a ^ flip)) ? 1u : 0u;
		T d = static_cast<T>(b - a);
		if (d >> (W - 1)) { d = static_cast<T>(T(0) - d); }
		bw_a = max(bw_a, bits_of(static_cast<uint64_t>(d)));
	}
	inc  = warp_sum(inc);
	dec  = warp_sum(dec);
	bw_a = warp_max(bw_a);
	// longest run: the run in progress entering each thread comes from a scan (original order) of
	// f(L) = (no start in the thread) ? L + 32 : length of the thread's last run
	const uint32_t u    = virtual_of_lane(lane);
	uint32_t       cont = sm == 0 ? 1u : 0u;
	uint32_t       cval = sm == 0 ? 32u : static_cast<uint32_t>(__clz(sm)) + 1u;
	{
		uint32_t a = __shfl_sync(0xFFFFFFFFu, cont, lane_of_virtual(lane));
		uint32_t c = __shfl_sync(0xFFFFFFFFu, cval, lane_of_virtual(lane));
#pragma unroll
		for (int d = 1; d < 32; d <<= 1) {
			const uint32_t pa = __shfl_up_sync(0xFFFFFFFFu, a, d);
			const uint32_t pc = __shfl_up_sync(0xFFFFFFFFu, c, d);
			if (lane >= static_cast<uint32_t>(d)) {
				c = a ? pc + c : c;
				a = pa & a;
			}
		}
		// virtual lane `lane` now holds the composition up to it; the run entering virtual u is that of u - 1
		const uint32_t entering_v = __shfl_up_sync(0xFFFFFFFFu, c, 1);
		const uint32_t ent        = __shfl_sync(0xFFFFFFFFu, lane == 0 ? 0u : entering_v, u);
		uint32_t       best       = 0;
		if (sm != 0) {
			const uint32_t head = static_cast<uint32_t>(__ffs(sm)) - 1u;
			best                = ent + head; // the run in progress ends at the first start (0 when nothing entered)
			int last            = -1;
#pragma unroll
			for (int i = 0; i < 32; ++i) {
				if ((sm >> i) & 1u) {
					if (last >= 0) { best = max(best, static_cast<uint32_t>(i - last)); }
					last = i;
				}
			}
		}
		if (u == 31) { best = max(best, sm == 0 ? ent + 32u : static_cast<uint32_t>(__clz(sm)) + 1u); }
		cval = warp_max(best);
	}
	const uint32_t maxrun = cval;
	// values with the top bit of (x - min) set, block ranges, zeros, min / max counts, magnitude
	T mnk = x[0] ^ flip, mxk = mnk;
#pragma unroll
	for (int i = 1; i < 32; ++i) {
		const T k = x[i] ^ flip;
		mnk       = k < mnk ? k : mnk;
		mxk       = k > mxk ? k : mxk;
	}
	const uint32_t blk = bits_of(static_cast<uint64_t>(static_cast<T>(mxk - mnk)));
	mnk                = warp_min(mnk);
	mxk                = warp_max(mxk);
	const T  mn = mnk ^ flip, mx = mxk ^ flip;
	uint32_t cnt_top = 0, nzero = 0, nmin = 0, nmax = 0, mag = 0;
#pragma unroll
	for (int i = 0; i < 32; ++i) {
		if (P.bw_f > 0) { cnt_top += static_cast<uint32_t>((static_cast<T>(x[i] - mn) >> (P.bw_f - 1)) & 1u); }
		nzero += x[i] == 0 ? 1u : 0u;
		nmin += x[i] == mn ? 1u : 0u;
		nmax += x[i] == mx ? 1u : 0u;
		T a = x[i];
		if (sgn && (a >> (W - 1))) { a = static_cast<T>(T(0) - a); }
		mag = max(mag, bits_of(static_cast<uint64_t>(a)));
	}
	cnt_top              = warp_sum(cnt_top);
	nzero                = warp_sum(nzero);
	nmin                 = warp_sum(nmin);
	nmax                 = warp_sum(nmax);
	mag                  = warp_max(mag);
	const uint32_t blk_s = warp_sum(blk);
	// lane f writes feature f
	const float    w = static_cast<float>(W), raw = 1024.0f * (W / 8), sz = static_cast<float>(W / 8);
	const float    r = static_cast<float>(P.runs), fdv = static_cast<float>(dv);
	const uint32_t cb = bits_of(dv - 1);
	float          f  = 0.0f;
	switch (lane) {
	case 0: f = P.bw_f / w; break;
	case 1: f = P.bw_d / w; break;
	case 2: f = r / 1024.0f; break;
	case 3: f = P.bw_i / 16.0f; break;
	case 4: f = fdv / 1024.0f; break;
	case 5: f = log2f(fdv) / 10.0f; break;
	case 6: f = cb / 16.0f; break;
	case 7: f = inc / 1023.0f; break;
	case 8: f = dec / 1023.0f; break;
	case 9: f = bw_a / w; break;
	case 10: f = maxrun / 1024.0f; break;
	case 11: f = log2f(1024.0f / r) / 10.0f; break;
	case 12: f = top / 1024.0f; break;
	case 13: f = cnt_top / 1024.0f; break;
	case 14: f = blk_s / (32.0f * w); break;
	case 15: f = w / 64.0f; break;
	case 16: f = sgn ? 1.0f : 0.0f; break;
	case 17: f = (1.0f + sz + 128.0f * P.bw_f) / raw; break;
	case 18: f = (129.0f + sz + 128.0f * P.bw_d) / raw; break;
	case 19: f = (r * sz + 131.0f + 128.0f * P.bw_i) / raw; break;
	case 20: f = (fdv * sz + 5.0f + 128.0f * cb) / raw; break;
	case 21: f = (fdv * sz + 4.0f * r + 131.0f + 128.0f * P.bw_i) / raw; break;
	case 22: f = mag / w; break;
	case 23: f = nzero / 1024.0f; break;
	case 24: f = fdv / r; break;
	case 25: f = log2f(static_cast<float>(maxrun)) / 10.0f; break;
	case 26: f = bits_of(top) / 11.0f; break;
	case 27: f = nmin / 1024.0f; break;
	case 28: f = nmax / 1024.0f; break;
	case 29: f = (static_cast<float>(P.bw_f) - blk_s / 32.0f) / w; break;
	case 30: f = P.bw_f == 0 ? 1.0f : 0.0f; break;
	default: f = dec == 0 ? 1.0f : 0.0f; break;
	}
	out[lane] = f;
}

// ---------------------------------------------------------------------------------------------------------
// Kernels over work items (warp per vector)
// ---------------------------------------------------------------------------------------------------------
struct ItemArgs {
	const Col*  cols;
	const Item* items;
	uint64_t    n_items;
};

__global__ void __launch_bounds__(kWarps * 32) k_parts(ItemArgs a, uint32_t* parts) {
	const uint32_t lane = threadIdx.x & 31u;
	for (uint64_t it = blockIdx.x * static_cast<uint64_t>(kWarps) + (threadIdx.x >> 5); it < a.n_items;
	     it += static_cast<uint64_t>(gridDim.x) * kWarps) {
		const Item m = a.items[it];
		const Col  c = a.cols[m.col];
		uint32_t   pk;
		if (c.width == 64) {
			uint64_t x[32];
			load_run<64>(c, m.vec, lane, x);
			pk = pack_parts(vector_parts<64>(x, lane, c.sgn != 0));
		} else {
			uint32_t x[32];
			load_run<32>(c, m.vec, lane, x);
			pk = pack_parts(vector_parts<32>(x, lane, c.sgn != 0));
		}
		if (lane == 0) { parts[it] = pk; }
	}
}

constexpr uint32_t kFeatSmem = kWarps * kHSlots * (8 + 4);

__global__ void __launch_bounds__(kWarps * 32) k_features(ItemArgs a, float* feat) {
	extern __shared__ __align__(16) uint8_t fsm[];
	const uint32_t lane = threadIdx.x & 31u, warp = threadIdx.x >> 5;
	uint64_t*      hk   = reinterpret_cast<uint64_t*>(fsm) + warp * kHSlots;
	uint32_t*      hc   = reinterpret_cast<uint32_t*>(fsm + kWarps * kHSlots * 8) + warp * kHSlots;
	for (uint32_t s = lane; s < kHSlots; s += 32) {
		hk[s] = kEmpty;
		hc[s] = 0;
	}
	__syncwarp();
	for (uint64_t it = blockIdx.x * static_cast<uint64_t>(kWarps) + warp; it < a.n_items;
	     it += static_cast<uint64_t>(gridDim.x) * kWarps) {
		const Item m = a.items[it];
		const Col  c = a.cols[m.col];
		if (c.width == 64) {
			uint64_t x[32];
			load_run<64>(c, m.vec, lane, x);
			const Parts P = vector_parts<64>(x, lane, c.sgn != 0);
			vector_features<64>(x, lane, c.sgn != 0, P, hk, hc, feat + it * NF);
		} else {
			uint32_t x[32];
			load_run<32>(c, m.vec, lane, x);
			const Parts P = vector_parts<32>(x, lane, c.sgn != 0);
			vector_features<32>(x, lane, c.sgn != 0, P, hk, hc, feat + it * NF);
		}
		__syncwarp();
	}
}

// ---------------------------------------------------------------------------------------------------------
// Dictionary of a chunk (wizard), one CTA per chunk: the chunk's distinct values, numbered in first-occurrence
// order (src/cor/lyt/dic/dic_fac.cpp:19-40), give the dictionary size and every vector's code bit width.
//   table     open addressing in shared memory (16 Ki slots), first position of every key by atomicMin.  A
//             chunk with more than kCdCap distinct values is split by hash into kCdParts buckets instead: one
//             read of the values scatters (key, position) pairs into the CTA's bucket scratch in global memory
//             (each bucket has room for the whole chunk), and every bucket (about 1/8 of the keys) goes
//             through the shared-memory table in turn, read back coalesced;
//   ranks     every key's first position sets a bit in the chunk's position bitmap (64 Ki bits, shared memory);
//             popcounts of the bitmap words, scanned, rank the first positions: a value's code;
//   codes     every value's code (the values again, or the buckets again), the code range of each vector.
// Exact for every chunk.
// ---------------------------------------------------------------------------------------------------------
constexpr uint32_t kCdSlots  = 1u << 14;
constexpr uint32_t kCdCap    = 12288; // distinct values the shared-memory table takes (a load of 3/4)
constexpr uint32_t kCdParts  = 8;     // buckets of a chunk of more distinct values (8 x 12288 > 65,536)
constexpr uint32_t kCdBucket = kMaxVecPerChunk * 1024;  // room of a bucket: the whole chunk
constexpr int      kCdWarps  = 16;
constexpr uint32_t kCdWords  = kMaxVecPerChunk * 1024 / 32;
constexpr uint32_t kCdSmem   = kCdSlots * 8 + (kCdSlots + 1) * 4 + 2 * kCdWords * 4 + 2 * kMaxVecPerChunk * 4;
constexpr uint64_t kCdGBytes = static_cast<uint64_t>(kCdParts) * kCdBucket * 12; // per CTA: keys, then positions
static_assert(kCdSmem <= 227 * 1024, "chunk dictionary tables fit one CTA");
static_assert(kMaxVecPerChunk <= 4 * kCdWarps, "at most 4 vectors of a chunk per warp");

struct ChunkDictArgs {
	const Col*      cols;
	const Item*     items;       // the chunks' vectors, chunk by chunk
	const uint32_t* chunk_items; // item range of every chunk (n_chunks + 1)
	uint32_t        n_chunks;
	uint32_t*       dict_n;  // per chunk: distinct values
	uint32_t*       bw_code; // per item: FFOR bit width of its codes
	int*            status;
	// string columns (optional): per-row weights of every column (row = vector * 1024 + position), summed over
	// the first occurrences of a chunk's distinct values into dict_w[chunk][0..1] (the dictionary's raw and
	// FSST-compressed bytes)
	const uint32_t* const* w0;
	const uint32_t* const* w1;
	uint64_t*       dict_w;
	uint8_t*        gtab; // gridDim.x regions of kCdGBytes: the CTAs' bucket scratch
};

// 64-bit finaliser of MurmurHash3 (Appleby): the slot from the low bits.
__device__ __forceinline__ uint64_t cd_mix(uint64_t x) {
	x ^= x >> 33;
	x *= 0xff51afd7ed558ccdull;
	x ^= x >> 33;
	x *= 0xc4ceb9fe1a85ec53ull;
	x ^= x >> 33;
	return x;
}

// Slot of x in a table of mask + 1 slots (inserted when absent; *count counts new keys): mask + 1 for the key
// ~0 (a slot of its own), mask + 2 when `limit` probes found neither x nor an empty slot.
__device__ __forceinline__ uint32_t cd_insert(uint64_t* keys, uint32_t mask, uint64_t x, uint32_t* count,
                                              uint32_t limit) {
	if (x == kEmpty) { return mask + 1; }
	uint32_t s = static_cast<uint32_t>(cd_mix(x)) & mask;
	for (uint32_t probe = 0; probe < limit; ++probe) {
		const uint64_t k = *reinterpret_cast<volatile uint64_t*>(keys + s);
		if (k == x) { return s; }
		if (k == kEmpty) {
			const uint64_t old = atomicCAS(reinterpret_cast<unsigned long long*>(keys + s), kEmpty, x);
			if (old == kEmpty) {
				atomicAdd(count, 1u);
				return s;
			}
			if (old == x) { return s; }
		}
		s = (s + 1) & mask;
	}
	return mask + 2;
}

__device__ __forceinline__ uint32_t cd_find(const uint64_t* keys, uint32_t mask, uint64_t x) {
	if (x == kEmpty) { return mask + 1; }
	uint32_t s = static_cast<uint32_t>(cd_mix(x)) & mask;
	for (uint32_t probe = 0; probe <= mask; ++probe) {
		const uint64_t k = keys[s];
		if (k == x) { return s; }
		if (k == kEmpty) { break; }
		s = (s + 1) & mask;
	}
	return mask + 2;
}

template <int W>
__device__ __forceinline__ void chunk_dict(const ChunkDictArgs& a, const Col& col, uint32_t c, uint64_t* keys,
                                           uint32_t* first, uint32_t* bits, uint32_t* pref, uint32_t* vrange,
                                           uint32_t* s_count, uint32_t* s_over, uint32_t* s_wsum, uint64_t* s_dw) {
	using T             = typename UT<W>::T;
	const uint32_t tid  = threadIdx.x, nt = blockDim.x, lane = tid & 31u, warp = tid >> 5, nw = nt >> 5;
	const uint32_t i0   = a.chunk_items[c], i1 = a.chunk_items[c + 1];
	const Item     m0   = a.items[i0];
	const uint32_t v0   = m0.vec - m0.cpos; // the chunk's first vector
	constexpr uint32_t mask = kCdSlots - 1;
	uint64_t* bkeys = reinterpret_cast<uint64_t*>(a.gtab + blockIdx.x * kCdGBytes);
	uint32_t* bpos  = reinterpret_cast<uint32_t*>(bkeys + static_cast<uint64_t>(kCdParts) * kCdBucket);
	auto begin_insert = [&]() {
		if (tid == 0) {
			*s_count = 0;
			*s_over  = 0;
		}
		__syncthreads();
	};
	// limit: probes before an insert gives up (the first attempt gives up early: its table must never fill,
	// or every insert into it walks all slots)
	auto insert_one = [&](uint64_t key, uint32_t pos, uint32_t limit) {
		const uint32_t sl = cd_insert(keys, mask, key, s_count, limit);
		if (sl > mask + 1) {
			*s_over = 1;
		} else if (pos < first[sl]) {
			atomicMin(first + sl, pos);
		}
	};
	auto clear_table = [&]() {
		for (uint32_t k = tid; k < kCdSlots; k += nt) { keys[k] = kEmpty; }
		for (uint32_t k = tid; k <= kCdSlots; k += nt) { first[k] = kNoPos; }
		__syncthreads();
	};
	// every key's first position into the bitmap (and, for strings, its row's weights); the table emptied
	auto harvest = [&]() {
		uint64_t sw0 = 0, sw1 = 0;
		for (uint32_t k = tid; k <= mask + 1; k += nt) {
			const uint32_t f = first[k];
			if (f != kNoPos) {
				atomicOr(bits + (f >> 5), 1u << (f & 31u));
				if (a.w0) {
					const uint64_t row = static_cast<uint64_t>(v0) * 1024 + f;
					sw0 += a.w0[m0.col][row];
					sw1 += a.w1[m0.col][row];
				}
			}
		}
		if (a.w0) {
			sw0 = warp_sum(sw0);
			sw1 = warp_sum(sw1);
			if (lane == 0) {
				atomicAdd(reinterpret_cast<unsigned long long*>(s_dw), static_cast<unsigned long long>(sw0));
				atomicAdd(reinterpret_cast<unsigned long long*>(s_dw + 1), static_cast<unsigned long long>(sw1));
			}
		}
		__syncthreads();
	};
	auto code_of = [&](uint32_t f) { return pref[f >> 5] + __popc(bits[f >> 5] & ((1u << (f & 31u)) - 1u)); };
	for (uint32_t k = tid; k < kCdWords; k += nt) { bits[k] = 0; }
	for (uint32_t k = tid; k < 2 * kMaxVecPerChunk; k += nt) { vrange[k] = (k & 1u) ? 0u : ~0u; }
	if (tid == 0) { s_dw[0] = s_dw[1] = 0; }
	// first attempt: every key of the chunk in the shared-memory table.  A thread stops within 4 inserts of
	// the count passing kCdCap (the table then holds at most kCdCap + 4 * 512 keys, 7/8 of its slots).
	begin_insert();
	volatile uint32_t* v_count = s_count;
	volatile uint32_t* v_over  = s_over;
	for (uint32_t j = i0 + warp; j < i1; j += nw) {
		if (*v_over != 0 || *v_count > kCdCap) { break; } // too many: the buckets instead
		const Item m = a.items[j];
		T          x[32];
		load_run<W>(col, m.vec, lane, x);
		const uint32_t pos0 = m.cpos * 1024 + thread_run(lane);
#pragma unroll
		for (int i = 0; i < 32; ++i) {
			if ((i & 3) == 0 && (*v_over != 0 || *v_count > kCdCap)) { break; }
			insert_one(static_cast<uint64_t>(x[i]), pos0 + i, 256);
		}
	}
	__syncthreads();
	const bool small = *s_over == 0 && *s_count <= kCdCap;
	__syncthreads();
	uint32_t bcount[kCdParts];
	if (small) {
		harvest();
	} else {
		clear_table();
		// one read of the values: (key, position) pairs into kCdParts buckets by hash
		if (tid < kCdParts) { s_wsum[tid] = 0; }
		__syncthreads();
		for (uint32_t j = i0 + warp; j < i1; j += nw) {
			const Item m = a.items[j];
			T          x[32];
			load_run<W>(col, m.vec, lane, x);
			const uint32_t pos0 = m.cpos * 1024 + thread_run(lane);
#pragma unroll
			for (int i = 0; i < 32; ++i) {
				const uint64_t key  = static_cast<uint64_t>(x[i]);
				const uint32_t b    = static_cast<uint32_t>(cd_mix(key) >> 61);
				const uint32_t peer = __match_any_sync(0xFFFFFFFFu, b);
				const uint32_t lead = __ffs(peer) - 1;
				uint32_t       base = 0;
				if (lane == lead) { base = atomicAdd(s_wsum + b, static_cast<uint32_t>(__popc(peer))); }
				base                 = __shfl_sync(peer, base, lead);
				const uint32_t slot  = base + __popc(peer & ((1u << lane) - 1u));
				const uint64_t where = static_cast<uint64_t>(b) * kCdBucket + slot;
				bkeys[where]         = key;
				bpos[where]          = pos0 + i;
			}
		}
		__syncthreads();
#pragma unroll
		for (uint32_t b = 0; b < kCdParts; ++b) { bcount[b] = s_wsum[b]; }
		__syncthreads();
		// every bucket through the table; once a bucket's table is complete, every pair's key is replaced by its
		// key's first position (high half) beside its own position, so the code pass needs no table
		for (uint32_t b = 0; b < kCdParts; ++b) {
			begin_insert();
			for (uint32_t k = tid; k < bcount[b]; k += nt) {
				const uint64_t where = static_cast<uint64_t>(b) * kCdBucket + k;
				insert_one(bkeys[where], bpos[where], kCdSlots);
			}
			__syncthreads();
			if ((*s_over != 0 || *s_count > mask) && tid == 0) { atomicOr(a.status, STATUS_BAD_INDEX); } // never
			for (uint32_t k = tid; k < bcount[b]; k += nt) {
				const uint64_t where = static_cast<uint64_t>(b) * kCdBucket + k;
				const uint32_t sl    = cd_find(keys, mask, bkeys[where]);
				const uint32_t f     = sl > mask + 1 ? kNoPos : first[sl];
				bkeys[where]         = (static_cast<uint64_t>(f) << 32) | bpos[where];
			}
			harvest(); // reads the table only; its closing barrier orders the clear after every find
			clear_table();
		}
	}
	// ranks: exclusive prefix of the bitmap words' popcounts (thread t: words [t * per, (t + 1) * per))
	const uint32_t per = kCdWords / nt;
	uint32_t       loc = 0;
	for (uint32_t k = 0; k < per; ++k) { loc += __popc(bits[tid * per + k]); }
	const uint32_t inc = warp_inclusive_scan(loc, lane);
	if (lane == 31) { s_wsum[warp] = inc; }
	__syncthreads();
	if (warp == 0) {
		const uint32_t w  = lane < nw ? s_wsum[lane] : 0u;
		const uint32_t wi = warp_inclusive_scan(w, lane);
		s_wsum[lane]      = wi - w;
		if (lane == 31) { s_wsum[32] = wi; }
	}
	__syncthreads();
	uint32_t run = s_wsum[warp] + inc - loc;
	for (uint32_t k = 0; k < per; ++k) {
		pref[tid * per + k] = run;
		run += __popc(bits[tid * per + k]);
	}
	const uint32_t total = s_wsum[32];
	__syncthreads();
	// codes: the code range of every vector of the chunk
	if (small) {
#pragma unroll
		for (uint32_t q = 0; q < 4; ++q) {
			const uint32_t j  = i0 + warp + q * nw;
			uint32_t       mn = ~0u, mx = 0u;
			if (j < i1) {
				const Item m = a.items[j];
				T          x[32];
				load_run<W>(col, m.vec, lane, x);
#pragma unroll
				for (int i = 0; i < 32; ++i) {
					const uint32_t sl = cd_find(keys, mask, static_cast<uint64_t>(x[i]));
					if (sl > mask + 1) { continue; }
					const uint32_t code = code_of(first[sl]);
					mn                  = min(mn, code);
					mx                  = max(mx, code);
				}
			}
			mn = warp_min(mn);
			mx = warp_max(mx);
			if (j < i1 && lane == 0) {
				vrange[2 * (j - i0)]     = mn;
				vrange[2 * (j - i0) + 1] = mx;
			}
		}
		__syncthreads();
		clear_table();
	} else {
		// codes from the recorded first positions; a warp whose pairs all belong to one vector (the usual case:
		// a bucket keeps the scatter's order) folds them before one atomic pair
		for (uint32_t b = 0; b < kCdParts; ++b) {
			for (uint32_t kb = 0; kb < bcount[b]; kb += nt) {
				const uint32_t k  = kb + tid;
				uint32_t       vi = ~0u, code = 0;
				if (k < bcount[b]) {
					const uint64_t e = bkeys[static_cast<uint64_t>(b) * kCdBucket + k];
					const uint32_t f = static_cast<uint32_t>(e >> 32);
					if (f != kNoPos) {
						vi   = static_cast<uint32_t>(e) >> 10; // the vector inside the chunk
						code = code_of(f);
					}
				}
				const uint32_t v0 = __shfl_sync(0xFFFFFFFFu, vi, 0);
				if (__all_sync(0xFFFFFFFFu, vi == v0)) {
					const uint32_t mn = warp_min(code), mx = warp_max(code);
					if (lane == 0 && v0 != ~0u) {
						atomicMin(vrange + 2 * v0, mn);
						atomicMax(vrange + 2 * v0 + 1, mx);
					}
				} else if (vi != ~0u) {
					atomicMin(vrange + 2 * vi, code);
					atomicMax(vrange + 2 * vi + 1, code);
				}
			}
		}
		__syncthreads();
	}
	for (uint32_t j = i0 + tid; j < i1; j += nt) {
		const uint32_t lo = vrange[2 * (j - i0)], hi = vrange[2 * (j - i0) + 1];
		a.bw_code[j]      = hi >= lo ? bits_of(hi - lo) : 0u;
	}
	if (tid == 0) {
		a.dict_n[c] = total;
		if (a.dict_w) {
			a.dict_w[2ull * c]     = s_dw[0];
			a.dict_w[2ull * c + 1] = s_dw[1];
		}
	}
	__syncthreads();
}

__global__ void __launch_bounds__(kCdWarps * 32) k_chunk_dict(ChunkDictArgs a) {
	extern __shared__ __align__(16) uint8_t smem[];
	__shared__ uint32_t s_count, s_over, s_wsum[33];
	__shared__ uint64_t s_dw[2];
	uint64_t*           keys   = reinterpret_cast<uint64_t*>(smem);
	uint32_t*           first  = reinterpret_cast<uint32_t*>(keys + kCdSlots);
	uint32_t*           bits   = first + kCdSlots + 1;
	uint32_t*           pref   = bits + kCdWords;
	uint32_t*           vrange = pref + kCdWords;
	for (uint32_t k = threadIdx.x; k < kCdSlots; k += blockDim.x) { keys[k] = kEmpty; }
	for (uint32_t k = threadIdx.x; k <= kCdSlots; k += blockDim.x) { first[k] = kNoPos; }
	__syncthreads();
	for (uint32_t c = blockIdx.x; c < a.n_chunks; c += gridDim.x) {
		const Col col = a.cols[a.items[a.chunk_items[c]].col];
		if (col.width == 64) {
			chunk_dict<64>(a, col, c, keys, first, bits, pref, vrange, &s_count, &s_over, s_wsum, s_dw);
		} else {
			chunk_dict<32>(a, col, c, keys, first, bits, pref, vrange, &s_count, &s_over, s_wsum, s_dw);
		}
	}
}

// ---------------------------------------------------------------------------------------------------------
// String columns.  The selection works on a 64-bit hash of every row (distinct rows, runs and first-occurrence
// codes come from the integer machinery run on the hashes), the row's length and its FSST-compressed length
// under the column's symbol table (the encoder's greedy longest match; a byte no symbol starts with costs an
// escape and itself, 2 bytes).  Candidates (string pool, no patches; src/cor/exp_pool.cpp:66-101):
//   0 BYTE_ARR (pool id 0)   1 DICT FFOR over an FSST dictionary (id 3)   2 FSST (id 13)
//   3 DICT_RLE with raw run codes and a raw u16 run index (id 15)
// ---------------------------------------------------------------------------------------------------------
constexpr int kStrK = FLS_SEL_STR_K;

// An FSST symbol table arranged for greedy matching: symbols grouped by their first byte, longest first.
struct StrTab {
	uint64_t val[256];
	uint8_t  len[256];
	uint16_t start[257]; // symbols starting with byte b: [start[b], start[b + 1])
};

struct StrCol {
	const uint8_t*  bytes;
	const uint64_t* offsets; // n_rows + 1
	uint64_t        n_bytes; // offsets[n_rows]
	const StrTab*   tab;
	uint32_t        tab_bytes; // the exported table's size (the FSST page's dictionary slot)
	uint64_t*       hash;      // per row
	uint32_t*       len;
	uint32_t*       clen;
};

__device__ __forceinline__ uint64_t str_mix(uint64_t h) {
	h ^= h >> 33;
	h *= 0xff51afd7ed558ccdull;
	h ^= h >> 33;
	h *= 0xc4ceb9fe1a85ec53ull;
	h ^= h >> 33;
	return h;
}

// 8 bytes of a string from byte position p (bytes past the column's last byte read as the last word's)
__device__ __forceinline__ uint64_t str_load8(const StrCol& c, uint64_t p) {
	const uint32_t* w    = reinterpret_cast<const uint32_t*>(reinterpret_cast<uintptr_t>(c.bytes) & ~uintptr_t(3));
	const uint64_t  a    = (reinterpret_cast<uintptr_t>(c.bytes) & 3u) + p; // byte index from w
	const uint64_t  last = ((reinterpret_cast<uintptr_t>(c.bytes) & 3u) + (c.n_bytes ? c.n_bytes - 1 : 0)) >> 2;
	const uint64_t  q    = a >> 2;
	const uint32_t  x0 = __ldg(w + (q < last ? q : last)), x1 = __ldg(w + (q + 1 < last ? q + 1 : last)),
	               x2  = __ldg(w + (q + 2 < last ? q + 2 : last));
	const uint32_t  sh = 8u * static_cast<uint32_t>(a & 3u);
	const uint32_t  lo = sh ? __funnelshift_r(x0, x1, sh) : x0, hi = sh ? __funnelshift_r(x1, x2, sh) : x1;
	return (static_cast<uint64_t>(hi) << 32) | lo;
}

// Block per item: hash and length of each of the vector's 1024 rows, and the compressed length of every rs-th
// row (rs = 1: every row, the exact figure the wizard's sizes need; rs > 1, the learned selector's features:
// the other rows' compressed lengths are written as 0 and the vector's sum is scaled by rs).  The column's
// symbol table is copied to shared memory for the greedy match; the vector's sums (vlen, vclen) by a block
// reduction.
__global__ void __launch_bounds__(kWarps * 32) k_str_rows(const StrCol* cols, const Item* items, uint64_t n_items,
                                                          uint64_t* vlen, uint64_t* vclen, uint32_t rs) {
	__shared__ uint64_t t_val[256];
	__shared__ uint8_t  t_len[256];
	__shared__ uint16_t t_start[257];
	__shared__ uint64_t red[2][kWarps];
	constexpr uint32_t  nt   = kWarps * 32;
	const uint32_t      tid  = threadIdx.x, lane = tid & 31u, warp = tid >> 5;
	for (uint64_t it = blockIdx.x; it < n_items; it += gridDim.x) {
		const Item   m = items[it];
		const StrCol c = cols[m.col];
		__syncthreads(); // the previous item's table reads and sums are done
		for (uint32_t k = tid; k < 257; k += nt) {
			if (k < 256) {
				t_val[k] = c.tab->val[k];
				t_len[k] = c.tab->len[k];
			}
			t_start[k] = c.tab->start[k];
		}
		__syncthreads();
		const uint64_t r0 = static_cast<uint64_t>(m.vec) * 1024;
		uint64_t       sl = 0, sc = 0;
		for (uint32_t j = tid; j < 1024; j += nt) {
			const uint64_t r = r0 + j;
			const uint64_t s = c.offsets[r], e = c.offsets[r + 1];
			const uint64_t n = e >= s ? e - s : 0;
			uint64_t       h = 0x243F6A8885A308D3ull ^ n;
			for (uint64_t p = 0; p < n; p += 8) {
				const uint64_t x = str_load8(c, s + p);
				const uint64_t k = n - p >= 8 ? x : (x & ((1ull << (8 * (n - p))) - 1));
				h                = str_mix(h ^ k) + 0x9E3779B97F4A7C15ull;
			}
			c.hash[r] = h;
			c.len[r]  = static_cast<uint32_t>(n);
			if (j % rs != 0) { c.clen[r] = 0; }
			sl += n;
		}
		// compressed lengths: rows rs * (tid + nt * i), spread over every thread
		for (uint32_t j = rs * tid; j < 1024; j += rs * nt) {
			const uint64_t r = r0 + j;
			const uint64_t s = c.offsets[r], e = c.offsets[r + 1];
			const uint64_t n = e >= s ? e - s : 0;
			uint64_t       cl = 0;
			for (uint64_t p = 0; p < n;) {
				const uint64_t x    = str_load8(c, s + p);
				const uint32_t b    = static_cast<uint32_t>(x & 0xFFu);
				const uint64_t left = n - p;
				uint32_t       step = 0;
				for (uint32_t k = t_start[b]; k < t_start[b + 1]; ++k) {
					const uint32_t l = t_len[k];
					if (l <= left && (l == 8 ? x : (x & ((1ull << (8 * l)) - 1))) == t_val[k]) {
						step = l;
						break;
					}
				}
				cl += step ? 1 : 2;
				p += step ? step : 1;
			}
			c.clen[r] = static_cast<uint32_t>(cl);
			sc += cl;
		}
		sl = warp_sum(sl);
		sc = warp_sum(sc);
		if (lane == 0) {
			red[0][warp] = sl;
			red[1][warp] = sc;
		}
		__syncthreads();
		if (tid == 0) {
			uint64_t a = 0, b = 0;
			for (int w = 0; w < kWarps; ++w) {
				a += red[0][w];
				b += red[1][w];
			}
			if (vlen) { vlen[it] = a; }
			if (vclen) { vclen[it] = b * rs; }
		}
	}
}

// blocks of k_str_rows (one item per block, at most 8 per SM)
int str_rows_grid(uint64_t n_items) {
	Device* d = current_device();
	if (!d) { return 0; }
	const uint64_t cap = static_cast<uint64_t>(d->sm_count) * 8;
	return static_cast<int>(std::max<uint64_t>(1, std::min<uint64_t>(n_items, cap)));
}

// The features of a string vector: those of its row hashes (distinct rows, runs, multiplicities), with the
// slots that mean nothing for hashes replaced by the rows' lengths and compressibility.
__global__ void __launch_bounds__(kWarps * 32) k_str_features(const StrCol* cols, const Item* items, uint64_t n_items,
                                                              float* feat, uint32_t rs) {
	const uint32_t lane = threadIdx.x & 31u;
	for (uint64_t it = blockIdx.x * static_cast<uint64_t>(kWarps) + (threadIdx.x >> 5); it < n_items;
	     it += static_cast<uint64_t>(gridDim.x) * kWarps) {
		const Item   m  = items[it];
		const StrCol c  = cols[m.col];
		float        sl = 0, sc = 0, sq = 0, mx = 0, mn = 1e30f;
		for (uint32_t i = 0; i < 32; ++i) {
			const uint64_t r = static_cast<uint64_t>(m.vec) * 1024 + lane + 32 * i;
			const float    l = static_cast<float>(c.len[r]);
			sl += l;
			sq += l * l;
			sc += static_cast<float>(c.clen[r]);
			mx = fmaxf(mx, l);
			mn = fminf(mn, l);
		}
		sl = warp_sum(sl);
		sq = warp_sum(sq);
		sc = warp_sum(sc) * static_cast<float>(rs); // every rs-th row's compressed length, scaled
		mx = warp_max(mx);
		mn = warp_min(mn);
		const float mean = sl / 1024.0f;
		const float var  = fmaxf(sq / 1024.0f - mean * mean, 0.0f);
		float*      f    = feat + it * NF;
		if (lane == 0) {
			f[0]  = mean / 64.0f;
			f[1]  = sl > 0 ? sc / sl : 1.0f;
			f[9]  = sqrtf(var) / 64.0f;
			f[14] = mx / 256.0f;
			f[15] = mn / 64.0f;
			f[16] = 1.0f; // a string column
			f[22] = log2f(mean + 1.0f) / 8.0f;
			f[29] = sc / (1024.0f * 64.0f);
		}
	}
}

struct StrSizeArgs {
	const uint32_t* chunk_col;
	const uint32_t* chunk_items; // item range of every chunk (n_chunks + 1)
	const uint32_t* parts;       // per item: runs of the row hashes in bits 19..
	const uint32_t* bw_code;     // per item
	const uint64_t* vlen;        // per item
	const uint64_t* vclen;       // per item
	const uint32_t* dict_n;      // per chunk
	const uint64_t* dict_w;      // per chunk: the dictionary's raw and compressed bytes
	const StrCol*   cols;
	uint32_t        n_chunks;
	uint64_t*       sizes; // n_chunks x FLS_SEL_K (the string candidates in 0..3, the rest ~0)
	uint8_t*        best;
};

// Exact page bytes of the string candidates (page = header, buffer offsets, per-vector entry points, buffers;
// the dictionary page of DICT and DICT_RLE = dict_hdr_t, the FSST_MAXHEADER table slot, u32 compressed lengths
// and the compressed entries, src/cor/lyt/dic/dic.cpp:88-111; the FSST column's = dict_hdr_t and the table).
__global__ void k_str_sizes(StrSizeArgs a) {
	const uint32_t lane = threadIdx.x & 31u;
	for (uint32_t c = blockIdx.x * (blockDim.x / 32) + (threadIdx.x >> 5); c < a.n_chunks; c += gridDim.x * (blockDim.x / 32)) {
		const uint32_t i0 = a.chunk_items[c], i1 = a.chunk_items[c + 1];
		uint64_t       L = 0, C = 0, R = 0, B = 0;
		for (uint32_t i = i0 + lane; i < i1; i += 32) {
			L += a.vlen[i];
			C += a.vclen[i];
			R += a.parts[i] >> 19;
			B += a.bw_code[i];
		}
		L = warp_sum(L), C = warp_sum(C), R = warp_sum(R), B = warp_sum(B);
		if (lane == 0) {
			const uint64_t nv    = i1 - i0;
			auto           frame = [&](uint64_t arr) { return 8 + 4 * arr + 4 * arr * (nv ? nv - 1 : 0); };
			const uint64_t dpage = 8 + 2066 + 4ull * a.dict_n[c] + a.dict_w[2ull * c + 1];
			uint64_t       z[FLS_SEL_K];
			z[0] = frame(2) + L + 4096 * nv;
			z[1] = frame(3) + nv + 4 * nv + 128 * B + dpage;
			z[2] = frame(2) + C + 4096 * nv + 8 + a.cols[a.chunk_col[c]].tab_bytes;
			z[3] = frame(2) + 4 * R + 2048 * nv + dpage;
			for (int k = kStrK; k < FLS_SEL_K; ++k) { z[k] = ~0ull; }
			uint32_t b = 0;
			for (int k = 0; k < FLS_SEL_K; ++k) {
				a.sizes[static_cast<uint64_t>(c) * FLS_SEL_K + k] = z[k];
				if (z[k] < z[b]) { b = k; }
			}
			a.best[c] = static_cast<uint8_t>(b);
		}
	}
}

// Exact sizes of every candidate of every chunk, and the smallest (lowest index on ties).
struct SizeArgs {
	const Col*      cols;
	const uint32_t* chunk_col;
	const uint32_t* chunk_items; // item range of every chunk (n_chunks + 1)
	const uint32_t* parts;       // per item
	const uint32_t* bw_code;     // per item
	const uint32_t* dict_n;      // per chunk
	uint32_t        n_chunks;
	uint64_t*       sizes;
	uint8_t*        best;
};

__global__ void k_chunk_sizes(SizeArgs a) {
	const uint32_t lane = threadIdx.x & 31u;
	for (uint32_t c = blockIdx.x * (blockDim.x / 32) + (threadIdx.x >> 5); c < a.n_chunks; c += gridDim.x * (blockDim.x / 32)) {
		const uint32_t i0 = a.chunk_items[c], i1 = a.chunk_items[c + 1];
		uint64_t       sf = 0, sd = 0, si = 0, sr = 0, sc = 0;
		for (uint32_t i = i0 + lane; i < i1; i += 32) {
			const uint32_t p = a.parts[i];
			sf += p & 127u;
			sd += (p >> 7) & 127u;
			si += (p >> 14) & 31u;
			sr += p >> 19;
			sc += a.bw_code[i];
		}
		sf = warp_sum(sf), sd = warp_sum(sd), si = warp_sum(si), sr = warp_sum(sr), sc = warp_sum(sc);
		if (lane == 0) {
			const uint64_t nv = i1 - i0, sz = a.cols[a.chunk_col[c]].width / 8;
			const uint64_t dp = 8 + 12 + static_cast<uint64_t>(a.dict_n[c]) * sz;
			uint64_t       s[K];
			s[0] = 8 + 4 * nv + 1024 * sz * nv;
			s[1] = 8 + 12 * nv + nv + sz * nv + 128 * sf;
			s[2] = 8 + 20 * nv + sz * sr + 128 * nv + nv + 2 * nv + 128 * si;
			s[3] = 8 + 16 * nv + 128 * nv + nv + sz * nv + 128 * sd;
			s[4] = dp + 8 + 12 * nv + nv + 4 * nv + 128 * sc;
			s[5] = dp + 8 + 20 * nv + 4 * sr + 128 * nv + nv + 2 * nv + 128 * si;
			uint32_t b = 0;
			for (int k = 0; k < K; ++k) {
				a.sizes[static_cast<uint64_t>(c) * K + k] = s[k];
				if (s[k] < s[b]) { b = k; }
			}
			a.best[c] = static_cast<uint8_t>(b);
		}
	}
}

// Per-chunk vote of the learned selector over its sampled rows: mean log-probability, argmax, mean top
// probability as the confidence.
__global__ void k_vote(const float* prob, const uint32_t* chunk_rows, uint32_t n_chunks, uint8_t* choice, float* conf,
                       int k_use) {
	const uint32_t lane = threadIdx.x & 31u;
	for (uint32_t c = blockIdx.x * (blockDim.x / 32) + (threadIdx.x >> 5); c < n_chunks; c += gridDim.x * (blockDim.x / 32)) {
		const uint32_t r0 = chunk_rows[c], r1 = chunk_rows[c + 1];
		float          lp[K] = {}, pp[K] = {};
		for (uint32_t r = r0 + lane; r < r1; r += 32) {
#pragma unroll
			for (int k = 0; k < K; ++k) {
				const float p = prob[static_cast<uint64_t>(r) * K + k];
				lp[k] += logf(fmaxf(p, 1e-30f));
				pp[k] += p;
			}
		}
		uint32_t b = 0;
#pragma unroll
		for (int k = 0; k < K; ++k) {
			lp[k] = warp_sum(lp[k]);
			pp[k] = warp_sum(pp[k]);
			if (k < k_use && lp[k] > lp[b]) { b = k; }
		}
		if (lane == 0) {
			choice[c] = static_cast<uint8_t>(b);
			if (conf) { conf[c] = r1 > r0 ? pp[b] / static_cast<float>(r1 - r0) : 0.0f; }
		}
	}
}

// ---------------------------------------------------------------------------------------------------------
// MLP kernels (float32)
// ---------------------------------------------------------------------------------------------------------
enum : int { EPI_NONE = 0, EPI_BIAS = 1, EPI_RELU = 2, EPI_MASK = 4 };

// C[M x N] = op(A)[M x Kd] * op(B)[Kd x N] with op = transpose when ta / tb; epilogue: + bias[n], ReLU, or
// zero where mask[m, n] <= 0 (the ReLU derivative).  64 x 64 tiles, 16-deep, 4 x 4 outputs per thread.
__global__ void __launch_bounds__(256) k_gemm(int M, int N, int Kd, const float* __restrict__ A, int lda, int ta,
                                              const float* __restrict__ B, int ldb, int tb, float* __restrict__ C,
                                              int ldc, const float* __restrict__ bias, const float* __restrict__ mask,
                                              int epi) {
	__shared__ float As[16][64 + 4];
	__shared__ float Bs[16][64 + 4];
	const int tx = threadIdx.x % 16, ty = threadIdx.x / 16;
	const int m0 = blockIdx.y * 64, n0 = blockIdx.x * 64;
	float     acc[4][4] = {};
	for (int k0 = 0; k0 < Kd; k0 += 16) {
		// consecutive threads walk the operand's contiguous dimension
		for (int e = threadIdx.x; e < 16 * 64; e += 256) {
			const int kk = ta ? e / 64 : e % 16, mm = ta ? e % 64 : e / 16;
			const int m = m0 + mm, k = k0 + kk;
			As[kk][mm]  = (m < M && k < Kd) ? (ta ? A[static_cast<int64_t>(k) * lda + m] : A[static_cast<int64_t>(m) * lda + k]) : 0.0f;
		}
		for (int e = threadIdx.x; e < 16 * 64; e += 256) {
			const int kk = tb ? e % 16 : e / 64, nn = tb ? e / 16 : e % 64;
			const int n = n0 + nn, k = k0 + kk;
			Bs[kk][nn]  = (n < N && k < Kd) ? (tb ? B[static_cast<int64_t>(n) * ldb + k] : B[static_cast<int64_t>(k) * ldb + n]) : 0.0f;
		}
		__syncthreads();
#pragma unroll
		for (int kk = 0; kk < 16; ++kk) {
			float a[4], b[4];
#pragma unroll
			for (int i = 0; i < 4; ++i) {
				a[i] = As[kk][ty + 16 * i];
				b[i] = Bs[kk][tx + 16 * i];
			}
#pragma unroll
			for (int i = 0; i < 4; ++i) {
#pragma unroll
				for (int j = 0; j < 4; ++j) { acc[i][j] = fmaf(a[i], b[j], acc[i][j]); }
			}
		}
		__syncthreads();
	}
#pragma unroll
	for (int i = 0; i < 4; ++i) {
		const int m = m0 + ty + 16 * i;
		if (m >= M) { continue; }
#pragma unroll
		for (int j = 0; j < 4; ++j) {
			const int n = n0 + tx + 16 * j;
			if (n >= N) { continue; }
			float v = acc[i][j];
			if (epi & EPI_BIAS) { v += bias[n]; }
			if (epi & EPI_RELU) { v = fmaxf(v, 0.0f); }
			if ((epi & EPI_MASK) && !(mask[static_cast<int64_t>(m) * ldc + n] > 0.0f)) { v = 0.0f; }
			C[static_cast<int64_t>(m) * ldc + n] = v;
		}
	}
}

// Softmax of every row of Z (n x K) into P; with labels: dZ = (P - onehot) / n and the mean loss added to
// *loss (and to loss_hist[*step] when given).
__global__ void k_softmax(const float* Z, uint64_t n, float* P, const int32_t* y, float* dZ, float* loss,
                          float* loss_hist, const uint32_t* step) {
	float l = 0.0f;
	for (uint64_t r = blockIdx.x * static_cast<uint64_t>(blockDim.x) + threadIdx.x; r < n;
	     r += static_cast<uint64_t>(gridDim.x) * blockDim.x) {
		float z[K], mx = -INFINITY, s = 0.0f;
#pragma unroll
		for (int k = 0; k < K; ++k) {
			z[k] = Z[r * K + k];
			mx   = fmaxf(mx, z[k]);
		}
#pragma unroll
		for (int k = 0; k < K; ++k) {
			z[k] = expf(z[k] - mx);
			s += z[k];
		}
#pragma unroll
		for (int k = 0; k < K; ++k) {
			z[k] /= s;
			if (P) { P[r * K + k] = z[k]; }
		}
		if (y) {
			const int32_t t = y[r];
			l -= logf(fmaxf(z[t], 1e-30f));
#pragma unroll
			for (int k = 0; k < K; ++k) { dZ[r * K + k] = (z[k] - (k == t ? 1.0f : 0.0f)) / static_cast<float>(n); }
		}
	}
	if (y) {
		l = warp_sum(l);
		if ((threadIdx.x & 31u) == 0) {
			if (loss) { atomicAdd(loss, l / static_cast<float>(n)); }
			if (loss_hist) { atomicAdd(loss_hist + *step, l / static_cast<float>(n)); }
		}
	}
}

// out[j] = sum over the n rows of X[r * ld + j] (bias gradients), one block per column.
__global__ void k_colsum(const float* X, uint64_t n, int cols, int ld, float* out) {
	__shared__ float ws[8];
	for (int j = blockIdx.x; j < cols; j += gridDim.x) {
		float s = 0.0f;
		for (uint64_t r = threadIdx.x; r < n; r += blockDim.x) { s += X[r * ld + j]; }
		s = warp_sum(s);
		if ((threadIdx.x & 31u) == 0) { ws[threadIdx.x >> 5] = s; }
		__syncthreads();
		if (threadIdx.x == 0) {
			float t = 0.0f;
			for (int w = 0; w < static_cast<int>(blockDim.x / 32); ++w) { t += ws[w]; }
			out[j] = t;
		}
		__syncthreads();
	}
}

// Adam (Kingma & Ba 2015, Algorithm 1); the step count comes from step_host, or from *step_dev + 1.
__global__ void k_adam(float* p, const float* g, float* m, float* v, uint64_t n, float lr, float b1, float b2,
                       float eps, uint32_t step_host, const uint32_t* step_dev) {
	const float t   = static_cast<float>(step_dev ? *step_dev + 1u : step_host);
	const float c1  = 1.0f - powf(b1, t);
	const float c2  = 1.0f - powf(b2, t);
	for (uint64_t i = blockIdx.x * static_cast<uint64_t>(blockDim.x) + threadIdx.x; i < n;
	     i += static_cast<uint64_t>(gridDim.x) * blockDim.x) {
		const float gi = g[i];
		const float mi = b1 * m[i] + (1.0f - b1) * gi;
		const float vi = b2 * v[i] + (1.0f - b2) * gi * gi;
		m[i]           = mi;
		v[i]           = vi;
		p[i] -= lr * (mi / c1) / (sqrtf(vi / c2) + eps);
	}
}

// Rows perm[step * B ..) of X / y into the contiguous batch.
__global__ void k_gather(const float* X, const int32_t* y, const uint32_t* perm, const uint32_t* step, uint32_t B,
                         float* Xb, int32_t* yb) {
	const uint64_t base = static_cast<uint64_t>(*step) * B;
	for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < B * NF; i += gridDim.x * blockDim.x) {
		const uint32_t r = i / NF, f = i % NF;
		const uint32_t src = perm[base + r];
		Xb[i]              = X[static_cast<uint64_t>(src) * NF + f];
		if (f == 0) { yb[r] = y[src]; }
	}
}

__global__ void k_step_inc(uint32_t* step) { ++*step; }

} // namespace sel
} // namespace flsgpu

// =========================================================================================================
// Host side
// =========================================================================================================
using namespace flsgpu;
using namespace flsgpu::sel;

namespace {

struct DevMem {
	void* p = nullptr;
	~DevMem() {
		if (p) { cudaFree(p); }
	}
	bool alloc(size_t n) {
		if (p) {
			cudaFree(p);
			p = nullptr;
		}
		return cudaMalloc(&p, n ? n : 1) == cudaSuccess;
	}
	template <class T>
	T* as() const {
		return static_cast<T*>(p);
	}
};

// Device scratch that only grows: a plan's calls reuse it instead of allocating (cudaFree synchronises the device).
struct Scratch {
	DevMem m;
	size_t cap = 0;
	bool   need(size_t n) {
		if (n <= cap && m.p) { return true; }
		if (!m.alloc(n)) {
			cap = 0;
			return false;
		}
		cap = n;
		return true;
	}
	template <class T>
	T* as() const {
		return m.as<T>();
	}
};

struct ItemSet {
	DevMem   items, chunk_items, row_chunk;
	uint64_t n = 0;
};

uint64_t param_count() { return NF * H + H + H * H + H + H * K + K; }

struct ParamView {
	const float *w1, *b1, *w2, *b2, *w3, *b3;
};
ParamView view(const float* p) {
	ParamView v;
	v.w1 = p;
	v.b1 = v.w1 + NF * H;
	v.w2 = v.b1 + H;
	v.b2 = v.w2 + H * H;
	v.w3 = v.b2 + H;
	v.b3 = v.w3 + H * K;
	return v;
}

cudaError_t gemm(cudaStream_t s, int M, int N, int Kd, const float* A, int lda, int ta, const float* B, int ldb, int tb,
                 float* C, int ldc, const float* bias, const float* mask, int epi) {
	if (M <= 0 || N <= 0) { return cudaSuccess; }
	// the grid's y extent is limited: tall row-major products go in slices of rows
	constexpr int kRows = 65535 * 64;
	if (M > kRows && ta) { return cudaErrorInvalidValue; }
	for (int m0 = 0; m0 < M; m0 += kRows) {
		const int  mm = std::min(kRows, M - m0);
		const dim3 grid((N + 63) / 64, (mm + 63) / 64);
		k_gemm<<<grid, 256, 0, s>>>(mm, N, Kd, A + static_cast<int64_t>(m0) * lda, lda, ta, B, ldb, tb,
		                            C + static_cast<int64_t>(m0) * ldc, ldc, bias,
		                            mask ? mask + static_cast<int64_t>(m0) * ldc : nullptr, epi);
		++launch_counter();
	}
	return cudaGetLastError();
}

// forward: H1, H2, Z of n rows
cudaError_t forward(cudaStream_t s, const float* params, const float* X, uint64_t n, float* H1, float* H2, float* Z) {
	const ParamView p = view(params);
	cudaError_t     e;
	if ((e = gemm(s, (int)n, H, NF, X, NF, 0, p.w1, H, 0, H1, H, p.b1, nullptr, EPI_BIAS | EPI_RELU)) != cudaSuccess) { return e; }
	if ((e = gemm(s, (int)n, H, H, H1, H, 0, p.w2, H, 0, H2, H, p.b2, nullptr, EPI_BIAS | EPI_RELU)) != cudaSuccess) { return e; }
	return gemm(s, (int)n, K, H, H2, H, 0, p.w3, K, 0, Z, K, p.b3, nullptr, EPI_BIAS);
}

// backward from dZ (n x K): gradients into G (parameter layout); dH2 / dH1: n x H scratch
cudaError_t backward(cudaStream_t s, const float* params, const float* X, uint64_t n, const float* H1, const float* H2,
                     const float* dZ, float* dH2, float* dH1, float* G) {
	const ParamView p = view(params);
	float*          gw1 = G;
	float*          gb1 = gw1 + NF * H;
	float*          gw2 = gb1 + H;
	float*          gb2 = gw2 + H * H;
	float*          gw3 = gb2 + H;
	float*          gb3 = gw3 + H * K;
	const int       nn  = static_cast<int>(n);
	cudaError_t     e;
	if ((e = gemm(s, H, K, nn, H2, H, 1, dZ, K, 0, gw3, K, nullptr, nullptr, EPI_NONE)) != cudaSuccess) { return e; }
	k_colsum<<<K, 256, 0, s>>>(dZ, n, K, K, gb3);
	++launch_counter();
	if ((e = gemm(s, nn, H, K, dZ, K, 0, p.w3, K, 1, dH2, H, nullptr, H2, EPI_MASK)) != cudaSuccess) { return e; }
	if ((e = gemm(s, H, H, nn, H1, H, 1, dH2, H, 0, gw2, H, nullptr, nullptr, EPI_NONE)) != cudaSuccess) { return e; }
	k_colsum<<<H, 256, 0, s>>>(dH2, n, H, H, gb2);
	++launch_counter();
	if ((e = gemm(s, nn, H, H, dH2, H, 0, p.w2, H, 1, dH1, H, nullptr, H1, EPI_MASK)) != cudaSuccess) { return e; }
	if ((e = gemm(s, NF, H, nn, X, NF, 1, dH1, H, 0, gw1, H, nullptr, nullptr, EPI_NONE)) != cudaSuccess) { return e; }
	k_colsum<<<H, 256, 0, s>>>(dH1, n, H, H, gb1);
	++launch_counter();
	return cudaGetLastError();
}

cudaError_t launch_features(const ItemArgs& a, float* feat, cudaStream_t s);

int grid_for(uint64_t warps_needed) {
	Device* d = current_device();
	if (!d) { return 0; }
	const uint64_t blocks = (warps_needed + kWarps - 1) / kWarps;
	const uint64_t cap    = static_cast<uint64_t>(d->sm_count) * 8;
	return static_cast<int>(std::max<uint64_t>(1, std::min(blocks, cap)));
}

cudaError_t launch_features(const ItemArgs& a, float* feat, cudaStream_t s) {
	static bool set = false;
	if (!set) {
		const cudaError_t e = cudaFuncSetAttribute(k_features, cudaFuncAttributeMaxDynamicSharedMemorySize, kFeatSmem);
		if (e != cudaSuccess) { return e; }
		set = true;
	}
	k_features<<<grid_for(a.n_items), kWarps * 32, kFeatSmem, s>>>(a, feat);
	++launch_counter();
	return cudaGetLastError();
}

__global__ void k_scatter_best(const uint8_t* best, const uint32_t* chunks, uint32_t n, uint8_t* out) {
	for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) { out[chunks[i]] = best[i]; }
}

} // namespace

struct fls_sel_plan {
	DevMem                cols_d, items_d, chunk_col_d, chunk_items_d;
	std::vector<Col>      cols;
	std::vector<Item>     items; // every vector, plan order
	std::vector<uint32_t> chunk_col, chunk_items;
	std::vector<uint64_t> chunk_first;
	uint64_t              n_chunks = 0;
	uint32_t              chunk_vectors = 64;
	// wizard scratch (gtab: the chunk dictionary's bucket scratch, one region per CTA; the subset lists of a
	// wizard run over some chunks) and the learned selector's; all grow-only
	Scratch bw_code, parts, dict_n, gtab, sub_items, sub_ranges, sub_ccol, sub_ids, sub_sizes, sub_best, vlen, vclen,
	    dict_w, l_work, l_conf;
	// string columns (fls_sel_plan_create_strings): the plan's columns are the row hashes; these are the strings
	bool                str = false;
	std::vector<StrCol> scols;
	DevMem              scols_d, tabs_d, hash_d, len_d, clen_d, wptr_d;
	std::map<uint32_t, ItemSet> samples; // stride -> sampled items
};

namespace {

int upload(DevMem& m, const void* h, size_t n) {
	if (!m.alloc(n)) { return FLS_ERR_CUDA; }
	if (n && cudaMemcpy(m.p, h, n, cudaMemcpyHostToDevice) != cudaSuccess) { return FLS_ERR_CUDA; }
	return FLS_OK;
}

// Sampled items (vectors 0, stride, ... of every chunk) with their chunk row ranges.
int sample_set(fls_sel_plan* p, uint32_t stride, ItemSet** out) {
	auto f = p->samples.find(stride);
	if (f == p->samples.end()) {
		std::vector<Item>     it;
		std::vector<uint32_t> rows(p->n_chunks + 1, 0), row_chunk;
		for (uint64_t c = 0; c < p->n_chunks; ++c) {
			rows[c] = static_cast<uint32_t>(it.size());
			for (uint32_t i = p->chunk_items[c]; i < p->chunk_items[c + 1]; i += stride) {
				it.push_back(p->items[i]);
				row_chunk.push_back(static_cast<uint32_t>(c));
			}
		}
		rows[p->n_chunks] = static_cast<uint32_t>(it.size());
		ItemSet& s        = p->samples[stride];
		s.n               = it.size();
		int rc;
		if ((rc = upload(s.items, it.data(), it.size() * sizeof(Item))) != FLS_OK) { return rc; }
		if ((rc = upload(s.chunk_items, rows.data(), rows.size() * 4)) != FLS_OK) { return rc; }
		if ((rc = upload(s.row_chunk, row_chunk.data(), row_chunk.size() * 4)) != FLS_OK) { return rc; }
		f = p->samples.find(stride);
	}
	*out = &f->second;
	return FLS_OK;
}

// Exact sizes of the chunks listed (all when chunks is empty).
int wizard_run(fls_sel_plan* p, const std::vector<uint32_t>& subset, uint64_t* d_sizes, uint8_t* d_best,
               uint32_t* d_dict_n, cudaStream_t s) {
	Device* dev = current_device();
	if (!dev) { return FLS_ERR_CUDA; }
	const bool            all = subset.empty();
	std::vector<uint32_t> chunks;
	if (all) {
		chunks.resize(p->n_chunks);
		for (uint64_t c = 0; c < p->n_chunks; ++c) { chunks[c] = static_cast<uint32_t>(c); }
	} else {
		chunks = subset;
	}
	// item list of the selected chunks (in chunk order) and their ranges: the plan's own device lists for all
	// chunks; for a subset, lists built here and copied in stream order into the plan's scratch
	const Item*     items_d  = p->items_d.as<Item>();
	const uint32_t* ranges_d = p->chunk_items_d.as<uint32_t>();
	const uint32_t* ccol_d   = p->chunk_col_d.as<uint32_t>();
	uint64_t        n_items  = p->items.size();
	if (!all) {
		std::vector<Item>     it;
		std::vector<uint32_t> ranges(chunks.size() + 1), ccol(chunks.size());
		for (size_t i = 0; i < chunks.size(); ++i) {
			const uint32_t c = chunks[i];
			ranges[i]        = static_cast<uint32_t>(it.size());
			ccol[i]          = p->chunk_col[c];
			for (uint32_t j = p->chunk_items[c]; j < p->chunk_items[c + 1]; ++j) {
				Item m  = p->items[j];
				m.chunk = static_cast<uint32_t>(i); // local chunk numbering for this run
				it.push_back(m);
			}
		}
		ranges[chunks.size()] = static_cast<uint32_t>(it.size());
		n_items               = it.size();
		if (it.empty()) { return FLS_OK; }
		if (!p->sub_items.need(it.size() * sizeof(Item)) || !p->sub_ranges.need(ranges.size() * 4) ||
		    !p->sub_ccol.need(ccol.size() * 4) || !p->sub_ids.need(chunks.size() * 4) ||
		    cudaMemcpyAsync(p->sub_items.m.p, it.data(), it.size() * sizeof(Item), cudaMemcpyHostToDevice, s) != cudaSuccess ||
		    cudaMemcpyAsync(p->sub_ranges.m.p, ranges.data(), ranges.size() * 4, cudaMemcpyHostToDevice, s) != cudaSuccess ||
		    cudaMemcpyAsync(p->sub_ccol.m.p, ccol.data(), ccol.size() * 4, cudaMemcpyHostToDevice, s) != cudaSuccess ||
		    cudaMemcpyAsync(p->sub_ids.m.p, chunks.data(), chunks.size() * 4, cudaMemcpyHostToDevice, s) != cudaSuccess ||
		    cudaStreamSynchronize(s) != cudaSuccess) { // the host lists go out of scope
			return FLS_ERR_CUDA;
		}
		items_d  = p->sub_items.as<Item>();
		ranges_d = p->sub_ranges.as<uint32_t>();
		ccol_d   = p->sub_ccol.as<uint32_t>();
	}
	if (n_items == 0) { return FLS_OK; }
	if (!p->parts.need(n_items * 4) || !p->bw_code.need(n_items * 4) || !p->dict_n.need(chunks.size() * 4)) {
		return FLS_ERR_CUDA;
	}
	if (p->str) {
		// the rows of every vector: hashes (the columns the integer passes read), lengths, compressed lengths
		if (!p->vlen.need(n_items * 8) || !p->vclen.need(n_items * 8) || !p->dict_w.need(chunks.size() * 16)) {
			return FLS_ERR_CUDA;
		}
		k_str_rows<<<str_rows_grid(n_items), kWarps * 32, 0, s>>>(p->scols_d.as<StrCol>(), items_d, n_items,
		                                                          p->vlen.as<uint64_t>(), p->vclen.as<uint64_t>(), 1u);
		++launch_counter();
	}
	ItemArgs ia {p->cols_d.as<Col>(), items_d, n_items};
	k_parts<<<grid_for(n_items), kWarps * 32, 0, s>>>(ia, p->parts.as<uint32_t>());
	++launch_counter();
	// dictionary of every chunk: one CTA per chunk, tables in shared memory
	{
		static bool attr[64] = {};
		if (dev->ordinal < 0 || dev->ordinal >= 64) { return FLS_ERR_CUDA; }
		if (!attr[dev->ordinal]) {
			if (cudaFuncSetAttribute(k_chunk_dict, cudaFuncAttributeMaxDynamicSharedMemorySize, kCdSmem) != cudaSuccess) {
				return FLS_ERR_CUDA;
			}
			attr[dev->ordinal] = true;
		}
		// one CTA per SM, each with its own bucket scratch for chunks of many distinct values
		const uint32_t grid = static_cast<uint32_t>(std::min<size_t>(chunks.size(), static_cast<size_t>(dev->sm_count)));
		if (!p->gtab.need(kCdGBytes * grid)) { return FLS_ERR_CUDA; }
		ChunkDictArgs a {p->cols_d.as<Col>(), items_d, ranges_d,
		                 static_cast<uint32_t>(chunks.size()), p->dict_n.as<uint32_t>(), p->bw_code.as<uint32_t>(),
		                 dev->status, nullptr, nullptr, nullptr, p->gtab.as<uint8_t>()};
		if (p->str) {
			const uint32_t* const* wp = p->wptr_d.as<const uint32_t*>();
			a.w0                      = wp;
			a.w1                      = wp + p->scols.size();
			a.dict_w                  = p->dict_w.as<uint64_t>();
		}
		k_chunk_dict<<<grid, kCdWarps * 32, kCdSmem, s>>>(a);
		++launch_counter();
		if (cudaGetLastError() != cudaSuccess) { return FLS_ERR_CUDA; }
	}
	uint64_t* sizes = d_sizes;
	uint8_t*  best  = d_best;
	if (!all) {
		if (!p->sub_sizes.need(chunks.size() * K * 8) || !p->sub_best.need(chunks.size())) { return FLS_ERR_CUDA; }
		sizes = p->sub_sizes.as<uint64_t>();
		best  = p->sub_best.as<uint8_t>();
	}
	if (p->str) {
		StrSizeArgs sa {ccol_d, ranges_d, p->parts.as<uint32_t>(), p->bw_code.as<uint32_t>(),
		                p->vlen.as<uint64_t>(), p->vclen.as<uint64_t>(), p->dict_n.as<uint32_t>(), p->dict_w.as<uint64_t>(),
		                p->scols_d.as<StrCol>(), static_cast<uint32_t>(chunks.size()), sizes, best};
		k_str_sizes<<<static_cast<unsigned>((chunks.size() + 7) / 8), 256, 0, s>>>(sa);
	} else {
		SizeArgs sa {p->cols_d.as<Col>(), ccol_d, ranges_d, p->parts.as<uint32_t>(),
		             p->bw_code.as<uint32_t>(), p->dict_n.as<uint32_t>(), static_cast<uint32_t>(chunks.size()), sizes, best};
		k_chunk_sizes<<<static_cast<unsigned>((chunks.size() + 7) / 8), 256, 0, s>>>(sa);
	}
	++launch_counter();
	if (cudaGetLastError() != cudaSuccess) { return FLS_ERR_CUDA; }
	if (!all) {
		// the subset's choices go to their chunks (sizes of a subset are not reported)
		if (d_best) {
			k_scatter_best<<<64, 256, 0, s>>>(best, p->sub_ids.as<uint32_t>(), static_cast<uint32_t>(chunks.size()), d_best);
			++launch_counter();
		}
	} else if (d_dict_n) {
		if (cudaMemcpyAsync(d_dict_n, p->dict_n.m.p, chunks.size() * 4, cudaMemcpyDeviceToDevice, s) != cudaSuccess) {
			return FLS_ERR_CUDA;
		}
	}
	return cudaStreamSynchronize(s) == cudaSuccess ? FLS_OK : FLS_ERR_CUDA;
}

} // namespace

extern "C" {

int fls_sel_plan_create(const fls_sel_column* cols, uint32_t n_cols, uint32_t chunk_vectors, fls_sel_plan** out) {
	if (!out || (!cols && n_cols) || chunk_vectors == 0 || chunk_vectors > kMaxVecPerChunk) { return FLS_ERR_ARG; }
	*out = nullptr;
	if (!current_device()) { return FLS_ERR_CUDA; }
	auto p           = std::make_unique<fls_sel_plan>();
	p->chunk_vectors = chunk_vectors;
	for (uint32_t c = 0; c < n_cols; ++c) {
		const fls_sel_column& s = cols[c];
		if ((s.width != 32 && s.width != 64) || (s.n_vec && !s.d_values) ||
		    (reinterpret_cast<uintptr_t>(s.d_values) & 15u) != 0 || s.n_vec >= (1ull << 32)) {
			return FLS_ERR_ARG;
		}
		p->cols.push_back(Col {static_cast<const uint8_t*>(s.d_values), s.n_vec, s.width, s.is_signed ? 1u : 0u});
		for (uint64_t v0 = 0; v0 < s.n_vec; v0 += chunk_vectors) {
			const uint32_t chunk = static_cast<uint32_t>(p->chunk_col.size());
			p->chunk_col.push_back(c);
			p->chunk_first.push_back(v0);
			p->chunk_items.push_back(static_cast<uint32_t>(p->items.size()));
			const uint64_t v1 = std::min<uint64_t>(s.n_vec, v0 + chunk_vectors);
			for (uint64_t v = v0; v < v1; ++v) {
				p->items.push_back(Item {c, chunk, static_cast<uint32_t>(v), static_cast<uint32_t>(v - v0)});
			}
		}
	}
	if (p->items.size() >= (1ull << 32)) { return FLS_ERR_TOO_LARGE; }
	p->n_chunks = p->chunk_col.size();
	p->chunk_items.push_back(static_cast<uint32_t>(p->items.size()));
	int rc;
	if ((rc = upload(p->cols_d, p->cols.data(), p->cols.size() * sizeof(Col))) != FLS_OK) { return rc; }
	if ((rc = upload(p->items_d, p->items.data(), p->items.size() * sizeof(Item))) != FLS_OK) { return rc; }
	if ((rc = upload(p->chunk_items_d, p->chunk_items.data(), p->chunk_items.size() * 4)) != FLS_OK) { return rc; }
	if ((rc = upload(p->chunk_col_d, p->chunk_col.data(), p->chunk_col.size() * 4)) != FLS_OK) { return rc; }
	*out = p.release();
	return FLS_OK;
}

} // extern "C"

namespace flsgpu {
int fsst_import_table(const uint8_t* buf, uint64_t avail, FsstTable* t, uint64_t* used);
}

namespace {
// An exported FSST table (fsst_export format) arranged for greedy matching: its symbols grouped by first byte,
// longest first (the codes past the table's symbol count, which decode as "corrupt", are not symbols).
int arrange_table(const uint8_t* tab, uint64_t n, StrTab* out) {
	FsstTable t {};
	const int rc = fsst_import_table(tab, n, &t, nullptr);
	if (rc != FLS_OK) { return rc; }
	const uint32_t zt = tab[8] & 1u;
	uint32_t       count = 0;
	for (uint32_t l = 0; l < 8; ++l) { count += tab[9 + l]; }
	if (zt && count) { --count; }
	std::vector<uint32_t> codes;
	for (uint32_t c = zt; c < zt + count && c < 255; ++c) { codes.push_back(c); }
	std::stable_sort(codes.begin(), codes.end(), [&](uint32_t x, uint32_t y) {
		const uint32_t bx = static_cast<uint32_t>(t.sym[x] & 0xFFu), by = static_cast<uint32_t>(t.sym[y] & 0xFFu);
		return bx != by ? bx < by : t.len[x] > t.len[y];
	});
	std::memset(out, 0, sizeof(*out));
	uint32_t k = 0;
	for (uint32_t b = 0; b < 256; ++b) {
		out->start[b] = static_cast<uint16_t>(k);
		while (k < codes.size() && (t.sym[codes[k]] & 0xFFu) == b) {
			out->val[k] = t.sym[codes[k]];
			out->len[k] = t.len[codes[k]];
			++k;
		}
	}
	out->start[256] = static_cast<uint16_t>(k);
	return FLS_OK;
}
} // namespace

extern "C" {

int fls_sel_plan_create_strings(const fls_sel_str_column* cols, uint32_t n_cols, uint32_t chunk_vectors,
                                fls_sel_plan** out) {
	if (!out || (!cols && n_cols)) { return FLS_ERR_ARG; }
	*out = nullptr;
	uint64_t rows = 0;
	for (uint32_t c = 0; c < n_cols; ++c) {
		if (cols[c].n_rows % 1024 || (cols[c].n_rows && (!cols[c].d_offsets || !cols[c].table)) ||
		    cols[c].n_rows >= (1ull << 41)) {
			return FLS_ERR_ARG;
		}
		rows += cols[c].n_rows;
	}
	DevMem hash, len, clen, tabs;
	if (!hash.alloc(rows * 8 + 16) || !len.alloc(rows * 4 + 16) || !clen.alloc(rows * 4 + 16) ||
	    !tabs.alloc(sizeof(StrTab) * (n_cols ? n_cols : 1))) {
		return FLS_ERR_CUDA;
	}
	// the plan's integer columns are the row hashes
	std::vector<fls_sel_column> hc(n_cols);
	std::vector<StrCol>         sc(n_cols);
	std::vector<StrTab>         st(n_cols);
	uint64_t                    r0 = 0;
	for (uint32_t c = 0; c < n_cols; ++c) {
		const fls_sel_str_column& x = cols[c];
		if (x.n_rows) {
			const int rc = arrange_table(x.table, x.table_size, &st[c]);
			if (rc != FLS_OK) { return rc; }
		}
		uint64_t nb = 0;
		if (x.n_rows && cudaMemcpy(&nb, x.d_offsets + x.n_rows, 8, cudaMemcpyDeviceToHost) != cudaSuccess) {
			return FLS_ERR_CUDA;
		}
		hc[c]          = fls_sel_column {};
		hc[c].d_values = hash.as<uint64_t>() + r0;
		hc[c].n_vec    = x.n_rows / 1024;
		hc[c].width    = 64;
		sc[c] = StrCol {x.d_bytes, x.d_offsets, nb, tabs.as<StrTab>() + c, static_cast<uint32_t>(x.table_size),
		                hash.as<uint64_t>() + r0, len.as<uint32_t>() + r0, clen.as<uint32_t>() + r0};
		r0 += x.n_rows;
	}
	fls_sel_plan* p  = nullptr;
	int           rc = fls_sel_plan_create(hc.data(), n_cols, chunk_vectors, &p);
	if (rc != FLS_OK) { return rc; }
	std::unique_ptr<fls_sel_plan> own(p);
	std::vector<const uint32_t*>  wp(2 * n_cols);
	for (uint32_t c = 0; c < n_cols; ++c) {
		wp[c]          = sc[c].len;
		wp[n_cols + c] = sc[c].clen;
	}
	if (n_cols && (cudaMemcpy(tabs.p, st.data(), sizeof(StrTab) * n_cols, cudaMemcpyHostToDevice) != cudaSuccess ||
	               (rc = upload(own->scols_d, sc.data(), sizeof(StrCol) * n_cols)) != FLS_OK ||
	               (rc = upload(own->wptr_d, wp.data(), sizeof(void*) * wp.size())) != FLS_OK)) {
		return rc != FLS_OK ? rc : FLS_ERR_CUDA;
	}
	own->str   = true;
	own->scols = sc;
	own->hash_d.p = hash.p, hash.p = nullptr;
	own->len_d.p  = len.p, len.p = nullptr;
	own->clen_d.p = clen.p, clen.p = nullptr;
	own->tabs_d.p = tabs.p, tabs.p = nullptr;
	*out          = own.release();
	return FLS_OK;
}

int fls_sel_plan_info(const fls_sel_plan* p, uint64_t* n_chunks, uint64_t* n_vectors) {
	if (!p) { return FLS_ERR_ARG; }
	if (n_chunks) { *n_chunks = p->n_chunks; }
	if (n_vectors) { *n_vectors = p->items.size(); }
	return FLS_OK;
}

int fls_sel_plan_chunks(const fls_sel_plan* p, uint32_t* h_col, uint64_t* h_first, uint32_t* h_count) {
	if (!p) { return FLS_ERR_ARG; }
	for (uint64_t c = 0; c < p->n_chunks; ++c) {
		if (h_col) { h_col[c] = p->chunk_col[c]; }
		if (h_first) { h_first[c] = p->chunk_first[c]; }
		if (h_count) { h_count[c] = p->chunk_items[c + 1] - p->chunk_items[c]; }
	}
	return FLS_OK;
}

int fls_sel_plan_destroy(fls_sel_plan* p) {
	delete p;
	return FLS_OK;
}

int fls_sel_vector_parts(const fls_sel_plan* p, uint32_t* d_parts, void* stream) {
	if (!p || (!d_parts && !p->items.empty())) { return FLS_ERR_ARG; }
	if (p->items.empty()) { return FLS_OK; }
	cudaStream_t s = static_cast<cudaStream_t>(stream);
	ItemArgs     a {p->cols_d.as<Col>(), p->items_d.as<Item>(), p->items.size()};
	k_parts<<<grid_for(p->items.size()), kWarps * 32, 0, s>>>(a, d_parts);
	++launch_counter();
	return cudaGetLastError() == cudaSuccess ? FLS_OK : FLS_ERR_CUDA;
}

int fls_sel_wizard(fls_sel_plan* p, uint64_t* d_sizes, uint8_t* d_best, uint32_t* d_dict_n, void* stream) {
	if (!p || ((!d_sizes || !d_best) && p->n_chunks)) { return FLS_ERR_ARG; }
	return wizard_run(p, {}, d_sizes, d_best, d_dict_n, static_cast<cudaStream_t>(stream));
}

} // extern "C"

namespace {
// Statistics of the items of a: for a string plan, the sampled vectors' rows first (hashes and lengths of every
// row, compressed lengths of every kStrFeatRowStride-th row), then the hash features with the string slots
// filled in.
constexpr uint32_t kStrFeatRowStride = 4;
cudaError_t        sample_features(fls_sel_plan* p, const ItemArgs& a, float* feat, cudaStream_t s) {
	if (p->str) {
		k_str_rows<<<str_rows_grid(a.n_items), kWarps * 32, 0, s>>>(p->scols_d.as<StrCol>(), a.items, a.n_items,
		                                                            nullptr, nullptr, kStrFeatRowStride);
		++launch_counter();
	}
	cudaError_t e = launch_features(a, feat, s);
	if (e != cudaSuccess || !p->str) { return e; }
	k_str_features<<<grid_for(a.n_items), kWarps * 32, 0, s>>>(p->scols_d.as<StrCol>(), a.items, a.n_items, feat,
	                                                           kStrFeatRowStride);
	++launch_counter();
	return cudaGetLastError();
}
} // namespace

extern "C" {

int fls_sel_features(fls_sel_plan* p, uint32_t stride, float* d_feat, uint32_t* d_row_chunk, uint64_t* n_rows,
                     void* stream) {
	if (!p || stride == 0 || !n_rows) { return FLS_ERR_ARG; }
	ItemSet* set = nullptr;
	int      rc  = sample_set(p, stride, &set);
	if (rc != FLS_OK) { return rc; }
	*n_rows = set->n;
	if (!d_feat || set->n == 0) { return FLS_OK; }
	cudaStream_t s = static_cast<cudaStream_t>(stream);
	ItemArgs     a {p->cols_d.as<Col>(), set->items.as<Item>(), set->n};
	if (sample_features(p, a, d_feat, s) != cudaSuccess) { return FLS_ERR_CUDA; }
	if (d_row_chunk && cudaMemcpyAsync(d_row_chunk, set->row_chunk.p, set->n * 4, cudaMemcpyDeviceToDevice, s) != cudaSuccess) {
		return FLS_ERR_CUDA;
	}
	return cudaGetLastError() == cudaSuccess ? FLS_OK : FLS_ERR_CUDA;
}

int fls_sel_learned(fls_sel_plan* p, const float* d_params, uint32_t stride, float threshold, uint8_t* d_choice,
                    float* d_conf, uint64_t* n_fallback, void* stream) {
	if (!p || !d_params || stride == 0 || (!d_choice && p->n_chunks)) { return FLS_ERR_ARG; }
	if (n_fallback) { *n_fallback = 0; }
	if (p->n_chunks == 0) { return FLS_OK; }
	cudaStream_t s   = static_cast<cudaStream_t>(stream);
	ItemSet*     set = nullptr;
	int          rc  = sample_set(p, stride, &set);
	if (rc != FLS_OK) { return rc; }
	const uint64_t n = set->n;
	if (!p->l_work.need(n * (NF + 2 * H + 2 * K) * 4) || !p->l_conf.need(p->n_chunks * 4)) { return FLS_ERR_CUDA; }
	Scratch& conf = p->l_conf;
	float*   feat = p->l_work.as<float>();
	float*   h1   = feat + n * NF;
	float*   h2   = h1 + n * H;
	float*   z    = h2 + n * H;
	float*   prob = z + n * K;
	ItemArgs a {p->cols_d.as<Col>(), set->items.as<Item>(), n};
	if (sample_features(p, a, feat, s) != cudaSuccess) { return FLS_ERR_CUDA; }
	if (forward(s, d_params, feat, n, h1, h2, z) != cudaSuccess) { return FLS_ERR_CUDA; }
	k_softmax<<<static_cast<unsigned>(std::min<uint64_t>((n + 255) / 256, 4096)), 256, 0, s>>>(z, n, prob, nullptr, nullptr,
	                                                                                            nullptr, nullptr, nullptr);
	k_vote<<<static_cast<unsigned>((p->n_chunks + 7) / 8), 256, 0, s>>>(prob, set->chunk_items.as<uint32_t>(),
	                                                                     static_cast<uint32_t>(p->n_chunks), d_choice,
	                                                                     conf.as<float>(), p->str ? kStrK : K);
	launch_counter() += 2;
	if (cudaGetLastError() != cudaSuccess) { return FLS_ERR_CUDA; }
	if (d_conf && cudaMemcpyAsync(d_conf, conf.m.p, p->n_chunks * 4, cudaMemcpyDeviceToDevice, s) != cudaSuccess) {
		return FLS_ERR_CUDA;
	}
	if (threshold > 0.0f) {
		std::vector<float> hc(p->n_chunks);
		if (cudaMemcpyAsync(hc.data(), conf.m.p, hc.size() * 4, cudaMemcpyDeviceToHost, s) != cudaSuccess ||
		    cudaStreamSynchronize(s) != cudaSuccess) {
			return FLS_ERR_CUDA;
		}
		std::vector<uint32_t> low;
		for (uint64_t c = 0; c < p->n_chunks; ++c) {
			if (hc[c] < threshold) { low.push_back(static_cast<uint32_t>(c)); }
		}
		if (n_fallback) { *n_fallback = low.size(); }
		if (!low.empty() && (rc = wizard_run(p, low, nullptr, d_choice, nullptr, s)) != FLS_OK) { return rc; }
	}
	return cudaStreamSynchronize(s) == cudaSuccess ? FLS_OK : FLS_ERR_CUDA;
}

uint64_t fls_sel_param_count(void) { return param_count(); }

int fls_sel_mlp_init(float* d_params, uint64_t seed) {
	if (!d_params) { return FLS_ERR_ARG; }
	std::vector<float>              h(param_count(), 0.0f);
	std::mt19937_64                 rng(seed);
	std::normal_distribution<float> nd(0.0f, 1.0f);
	float*                          w1 = h.data();
	float*                          w2 = w1 + NF * H + H;
	float*                          w3 = w2 + H * H + H;
	for (int i = 0; i < NF * H; ++i) { w1[i] = nd(rng) * std::sqrt(2.0f / NF); }
	for (int i = 0; i < H * H; ++i) { w2[i] = nd(rng) * std::sqrt(2.0f / H); }
	for (int i = 0; i < H * K; ++i) { w3[i] = nd(rng) * std::sqrt(2.0f / H); }
	return cudaMemcpy(d_params, h.data(), h.size() * 4, cudaMemcpyHostToDevice) == cudaSuccess ? FLS_OK : FLS_ERR_CUDA;
}

int fls_sel_mlp_forward(const float* d_params, const float* d_x, uint64_t n, float* d_prob, void* stream) {
	if (!d_params || ((!d_x || !d_prob) && n) || n >= (1ull << 31)) { return FLS_ERR_ARG; }
	if (n == 0) { return FLS_OK; }
	cudaStream_t s = static_cast<cudaStream_t>(stream);
	DevMem       w;
	if (!w.alloc(n * (2 * H + K) * 4)) { return FLS_ERR_CUDA; }
	float* h1 = w.as<float>();
	float* h2 = h1 + n * H;
	float* z  = h2 + n * H;
	if (forward(s, d_params, d_x, n, h1, h2, z) != cudaSuccess) { return FLS_ERR_CUDA; }
	k_softmax<<<static_cast<unsigned>(std::min<uint64_t>((n + 255) / 256, 4096)), 256, 0, s>>>(z, n, d_prob, nullptr, nullptr,
	                                                                                            nullptr, nullptr, nullptr);
	++launch_counter();
	return cudaStreamSynchronize(s) == cudaSuccess ? FLS_OK : FLS_ERR_CUDA;
}

int fls_sel_mlp_grad(const float* d_params, const float* d_x, const int32_t* d_y, uint64_t n, float* d_grad,
                     float* d_loss, void* stream) {
	if (!d_params || !d_x || !d_y || !d_grad || !d_loss || n == 0 || n >= (1ull << 31)) { return FLS_ERR_ARG; }
	cudaStream_t s = static_cast<cudaStream_t>(stream);
	DevMem       w;
	if (!w.alloc(n * (4 * H + 2 * K) * 4)) { return FLS_ERR_CUDA; }
	float* h1  = w.as<float>();
	float* h2  = h1 + n * H;
	float* z   = h2 + n * H;
	float* dz  = z + n * K;
	float* dh2 = dz + n * K;
	float* dh1 = dh2 + n * H;
	if (cudaMemsetAsync(d_loss, 0, 4, s) != cudaSuccess) { return FLS_ERR_CUDA; }
	if (forward(s, d_params, d_x, n, h1, h2, z) != cudaSuccess) { return FLS_ERR_CUDA; }
	k_softmax<<<static_cast<unsigned>(std::min<uint64_t>((n + 255) / 256, 4096)), 256, 0, s>>>(z, n, nullptr, d_y, dz, d_loss,
	                                                                                            nullptr, nullptr);
	++launch_counter();
	if (backward(s, d_params, d_x, n, h1, h2, dz, dh2, dh1, d_grad) != cudaSuccess) { return FLS_ERR_CUDA; }
	return cudaStreamSynchronize(s) == cudaSuccess ? FLS_OK : FLS_ERR_CUDA;
}

int fls_sel_adam_step(float* d_params, const float* d_grad, float* d_m, float* d_v, float lr, float beta1, float beta2,
                      float eps, uint32_t step, void* stream) {
	if (!d_params || !d_grad || !d_m || !d_v || step == 0) { return FLS_ERR_ARG; }
	cudaStream_t s = static_cast<cudaStream_t>(stream);
	k_adam<<<64, 256, 0, s>>>(d_params, d_grad, d_m, d_v, param_count(), lr, beta1, beta2, eps, step, nullptr);
	++launch_counter();
	return cudaGetLastError() == cudaSuccess ? FLS_OK : FLS_ERR_CUDA;
}

int fls_sel_train(float* d_params, const float* d_x, const int32_t* d_y, const uint32_t* d_perm, uint32_t batch,
                  uint32_t steps, float lr, float* d_loss_hist, void* stream) {
	if (!d_params || !d_x || !d_y || !d_perm || batch == 0 || batch > (1u << 20)) { return FLS_ERR_ARG; }
	if (steps == 0) { return FLS_OK; }
	// capture needs a stream other than the legacy default one: a private stream ordered after the caller's
	cudaStream_t caller = static_cast<cudaStream_t>(stream);
	cudaStream_t s      = nullptr;
	cudaEvent_t  ev     = nullptr;
	if (cudaStreamCreateWithFlags(&s, cudaStreamNonBlocking) != cudaSuccess) { return FLS_ERR_CUDA; }
	struct Guard {
		cudaStream_t s;
		cudaEvent_t* ev;
		~Guard() {
			if (*ev) { cudaEventDestroy(*ev); }
			cudaStreamSynchronize(s);
			cudaStreamDestroy(s);
		}
	} guard {s, &ev};
	if (cudaEventCreateWithFlags(&ev, cudaEventDisableTiming) != cudaSuccess || cudaEventRecord(ev, caller) != cudaSuccess ||
	    cudaStreamWaitEvent(s, ev, 0) != cudaSuccess) {
		return FLS_ERR_CUDA;
	}
	const uint64_t P = param_count(), B = batch;
	DevMem         w;
	if (!w.alloc((B * (NF + 4 * H + 2 * K) + 3 * P) * 4 + B * 4 + 64)) { return FLS_ERR_CUDA; }
	float*    xb  = w.as<float>();
	float*    h1  = xb + B * NF;
	float*    h2  = h1 + B * H;
	float*    z   = h2 + B * H;
	float*    dz  = z + B * K;
	float*    dh2 = dz + B * K;
	float*    dh1 = dh2 + B * H;
	float*    g   = dh1 + B * H;
	float*    m   = g + P;
	float*    v   = m + P;
	int32_t*  yb  = reinterpret_cast<int32_t*>(v + P);
	uint32_t* st  = reinterpret_cast<uint32_t*>(yb + B);
	if (cudaMemsetAsync(m, 0, 2 * P * 4, s) != cudaSuccess || cudaMemsetAsync(st, 0, 4, s) != cudaSuccess) {
		return FLS_ERR_CUDA;
	}
	if (d_loss_hist && cudaMemsetAsync(d_loss_hist, 0, steps * 4ull, s) != cudaSuccess) { return FLS_ERR_CUDA; }
	// one training step, captured once and replayed `steps` times
	cudaGraph_t     graph = nullptr;
	cudaGraphExec_t exec  = nullptr;
	const uint64_t launches0 = launch_counter();
	if (cudaStreamBeginCapture(s, cudaStreamCaptureModeThreadLocal) != cudaSuccess) { return FLS_ERR_CUDA; }
	k_gather<<<64, 256, 0, s>>>(d_x, d_y, d_perm, st, batch, xb, yb);
	forward(s, d_params, xb, B, h1, h2, z);
	k_softmax<<<static_cast<unsigned>((B + 255) / 256), 256, 0, s>>>(z, B, nullptr, yb, dz, nullptr, d_loss_hist, st);
	backward(s, d_params, xb, B, h1, h2, dz, dh2, dh1, g);
	k_adam<<<64, 256, 0, s>>>(d_params, g, m, v, P, lr, 0.9f, 0.999f, 1e-8f, 0, st);
	k_step_inc<<<1, 1, 0, s>>>(st);
	const cudaError_t ce = cudaStreamEndCapture(s, &graph);
	launch_counter()     = launches0;
	if (ce != cudaSuccess || !graph) { return FLS_ERR_CUDA; }
	const cudaError_t ie = cudaGraphInstantiate(&exec, graph, 0);
	cudaGraphDestroy(graph);
	if (ie != cudaSuccess) { return FLS_ERR_CUDA; }
	int rc = FLS_OK;
	for (uint32_t i = 0; i < steps && rc == FLS_OK; ++i) {
		if (cudaGraphLaunch(exec, s) != cudaSuccess) { rc = FLS_ERR_CUDA; }
	}
	launch_counter() += static_cast<uint64_t>(steps) * 15; // kernels per replayed step
	if (cudaStreamSynchronize(s) != cudaSuccess) { rc = FLS_ERR_CUDA; }
	cudaGraphExecDestroy(exec);
	return rc;
}

} // extern "C"
