// The B200 decode engine: one persistent kernel that walks a queue of (column, vector) work items and decodes
// each FastLanes vector with one warp.
//
//   stage 1  packed words of the vector -> shared memory with a bulk TMA copy (cp.async.bulk + mbarrier),
//            STAGES vectors ahead of the one being decoded (per-warp ring)
//   stage 2  bit-unpack + FOR add (+ per-lane running sum for DELTA) in registers, values in run order
//   stage 3  optional gather: RLE expansion from the run values staged next to the packed words, or a
//            dictionary lookup
//   stage 4  store: transposed order straight from registers, original order through a swizzled staging
//            buffer and row-wise 16-byte stores (every decoded byte crosses HBM exactly once)
//
// Reference semantics (cwida/FastLanes): unpack/unffor = primitives/fls_generated/fallback/scalar_aav_uf1/
// *_unpack_src.cpp:17277 / *_unffor_src.cpp:22971 (u32 dispatch), rsum = *_rsum_src.cpp:100-410,
// untranspose_i = *_untranspose_src.cpp:4110, RLE expansion = src/cor/lyt/vec.cpp:318-332 (Vec::flatten_to),
// dictionary gather = include/fls/encoder/assert_eq.hpp:257-400.
#include "fls_device.cuh"
#include "fls_plan.h"

namespace flsgpu {

struct Plan {
	const uint8_t* src;        // packed words of the stream
	const uint8_t* lane_bases; // ENC_DELTA
	const uint8_t* gsrc;       // RLE run values
	const uint8_t* dict;
	uint8_t*       out;
	uint64_t       for_base;
	uint32_t       bytes;  // packed bytes = bw * 128
	uint32_t       gbytes; // run-value bytes
	uint32_t       bw;
	uint32_t       entry_c;
	uint32_t       n_runs;
	uint32_t       ghead; // offset of the run values inside the staged (16-byte aligned) copy
	uint8_t        ws, e, enc, post, order;
	uint8_t        cmp; // OUT_BITMAP_* of filter plans, else OUT_VALUES
	bool           ok;
	bool           lb_exact; // lane bases outside a page: copy exactly 128 bytes, never a window around them
};

__device__ __forceinline__ uint64_t ld_le(const uint8_t* p, uint32_t n) {
	const uintptr_t a = reinterpret_cast<uintptr_t>(p);
	if ((a & (n - 1)) == 0) {
		switch (n) {
		case 1: return *p;
		case 2: return *reinterpret_cast<const uint16_t*>(p);
		case 4: return *reinterpret_cast<const uint32_t*>(p);
		default: return *reinterpret_cast<const uint64_t*>(p);
		}
	}
	if (n == 8 && (a & 3u) == 0) {
		const uint32_t* w = reinterpret_cast<const uint32_t*>(p);
		return static_cast<uint64_t>(w[0]) | (static_cast<uint64_t>(w[1]) << 32);
	}
	uint64_t x = 0;
	for (uint32_t i = 0; i < n; ++i) { x |= static_cast<uint64_t>(p[i]) << (8 * i); }
	return x;
}

// Entry points sit at page offset 8 + 4*arr_c; a page may be placed at any byte address (it is placed so that
// its packed buffer is 16-byte aligned), so they are read alignment-agnostically.
// Little-endian load of 4 / 8 bytes at any byte address inside a shared-memory staging area that has at least 8
// readable bytes after it: aligned words joined by funnel shifts instead of byte loads.
__device__ __forceinline__ uint32_t sld4(const uint8_t* p) {
	const uintptr_t a = reinterpret_cast<uintptr_t>(p);
	const uint32_t* w = reinterpret_cast<const uint32_t*>(a & ~uintptr_t(3));
	return (a & 3u) ? __funnelshift_r(w[0], w[1], (a & 3u) * 8u) : w[0];
}
__device__ __forceinline__ uint64_t sld8(const uint8_t* p) {
	const uintptr_t a = reinterpret_cast<uintptr_t>(p);
	const uint32_t* w = reinterpret_cast<const uint32_t*>(a & ~uintptr_t(3));
	const uint32_t  s = (a & 3u) * 8u;
	const uint32_t  lo = s ? __funnelshift_r(w[0], w[1], s) : w[0];
	const uint32_t  hi = s ? __funnelshift_r(w[1], w[2], s) : w[1];
	return (static_cast<uint64_t>(hi) << 32) | lo;
}
template <int E>
__device__ __forceinline__ uint64_t sld(const uint8_t* p) {
	if constexpr (E == 8) {
		return sld8(p);
	} else if constexpr (E == 4) {
		return sld4(p);
	} else {
		return ld_le(p, E);
	}
}

__device__ __forceinline__ uint32_t ep_of(const ColDesc& c, uint32_t v, uint32_t i) {
	if (v == 0) { return 0u; }
	return static_cast<uint32_t>(ld_le(reinterpret_cast<const uint8_t*>(c.ep) + 4ull * ((v - 1) * c.arr_c + i), 4));
}

__device__ __forceinline__ Plan make_plan(const ColDesc& c, uint32_t v) {
	Plan p;
	p.ws      = c.ws;
	p.e       = c.e;
	p.enc     = c.enc;
	p.post    = c.post;
	p.order   = c.order;
	p.entry_c = c.entry_c;
	p.dict    = c.dict;
	p.cmp     = c.out_mode;
	p.out     = c.out + static_cast<uint64_t>(v) * (c.out_mode != OUT_VALUES ? 128u : kVec * c.e);
	p.ok      = v < c.n_vec;
	p.lb_exact   = c.layout == LAYOUT_ARRAYS;
	p.for_base   = 0;
	p.lane_bases = nullptr;
	p.gsrc       = nullptr;
	p.gbytes     = 0;
	p.n_runs     = 0;
	p.ghead      = 0;
	const uint32_t wb = c.ws / 8;
	if (c.layout == LAYOUT_ARRAYS) {
		p.bw               = c.bw_arr ? c.bw_arr[v] : c.bw_const;
		const uint64_t off = c.byte_off ? c.byte_off[v] : static_cast<uint64_t>(v) * c.bw_const * 128u;
		p.src              = c.packed + off;
		if (c.base_arr) { p.for_base = ld_le(c.base_arr + static_cast<uint64_t>(v) * wb, wb); }
		if (c.lane_base_arr) { p.lane_bases = c.lane_base_arr + static_cast<uint64_t>(v) * 128u; }
	} else {
		if (c.enc == ENC_RAW) {
			p.bw = c.ws;
		} else {
			const uint32_t obw = ep_of(c, v, c.ib_bw);
			const uint32_t obs = ep_of(c, v, c.ib_base);
			if (obw >= c.buf_size[c.ib_bw] || obs + wb > c.buf_size[c.ib_base]) { p.ok = false; }
			p.bw       = p.ok ? c.buf[c.ib_bw][obw] : 0;
			p.for_base = p.ok ? ld_le(c.buf[c.ib_base] + obs, wb) : 0;
		}
		const uint32_t opk = ep_of(c, v, c.ib_packed);
		p.src              = c.buf[c.ib_packed] + opk;
		if (static_cast<uint64_t>(opk) + p.bw * 128ull > c.buf_size[c.ib_packed]) { p.ok = false; }
		if (c.enc == ENC_DELTA) {
			const uint32_t olb = ep_of(c, v, c.ib_lane_bases);
			if (olb + 128ull > c.buf_size[c.ib_lane_bases]) { p.ok = false; }
			p.lane_bases = c.buf[c.ib_lane_bases] + olb;
		}
		if (post_is_patch(c.post)) {
			// exceptions (gsrc, gbytes) and their positions / bitmap / chain head (dict, entry_c bytes)
			const uint32_t oe = ep_of(c, v, c.ib_exc), os = ep_of(c, v, c.ib_side);
			const uint64_t ee = (v + 1 < c.n_vec) ? ep_of(c, v + 1, c.ib_exc) : c.buf_size[c.ib_exc];
			const uint64_t es = (v + 1 < c.n_vec) ? ep_of(c, v + 1, c.ib_side) : c.buf_size[c.ib_side];
			if (ee < oe || ee > c.buf_size[c.ib_exc] || es < os || es > c.buf_size[c.ib_side]) { p.ok = false; }
			p.gsrc    = c.buf[c.ib_exc] + oe;
			p.gbytes  = p.ok ? static_cast<uint32_t>(ee - oe) : 0u;
			p.dict    = c.buf[c.ib_side] + os;
			p.entry_c = p.ok ? static_cast<uint32_t>(es - os) : 0u;
		}
		if (c.post == POST_RLE || c.post == POST_RLE_DICT) {
			const uint32_t ov  = ep_of(c, v, c.ib_vals);
			const uint64_t end = (v + 1 < c.n_vec) ? ep_of(c, v + 1, c.ib_vals) : c.buf_size[c.ib_vals];
			if (end < ov || end > c.buf_size[c.ib_vals]) { p.ok = false; }
			p.gsrc   = c.buf[c.ib_vals] + ov;
			p.gbytes = p.ok ? static_cast<uint32_t>(end - ov) : 0;
		}
	}
	if (p.bw > p.ws) { p.ok = false; }
	p.bytes = p.ok ? p.bw * 128u : 0u;
	if (p.post == POST_RLE || p.post == POST_RLE_DICT) {
		const uint32_t ve = p.post == POST_RLE ? p.e : 4u;
		if (p.gbytes > kVec * ve) { p.ok = false; }
		p.n_runs = p.ok ? p.gbytes / ve : 0u;
		p.ghead  = static_cast<uint32_t>(reinterpret_cast<uintptr_t>(p.gsrc) & 15u);
	}
	return p;
}

#ifndef FLS_HOST_EMULATION
// Copy one vector's inputs into its stage and arm the stage's mbarrier.  Called by all 32 lanes with the same
// plan.  16-byte aligned packed words go through the TMA engine; anything else is copied by the warp.
// The run values of an RLE vector are fetched as the enclosing 16-byte aligned window (pages are placed
// with at least 16 bytes of slack on both sides), so they always take the TMA path.
// The 128 lane bases of a DELTA vector travel with its packed words: the 16-byte aligned window around them
// (at most 144 bytes, inside the page) lands in a per-slot area of kLaneWindow bytes.
constexpr uint32_t kLaneWindow = 256;

template <uint32_t GSTAGE>
__device__ __forceinline__ void issue(const Plan& p, uint8_t* stage, uint8_t* gstage, uint8_t* lbstage, uint64_t* bar,
                                      uint32_t lane, bool stall = false) {
	uint32_t       tx     = 0;
	const uint32_t lbhead = static_cast<uint32_t>(reinterpret_cast<uintptr_t>(p.lane_bases) & 15u);
	// 16-byte aligned lane bases: exactly their 128 bytes by TMA; inside a page: the aligned 144-byte window by
	// TMA; otherwise (a misaligned caller array) the warp copies the 128 bytes
	const bool lbtma  = p.ok && p.lane_bases != nullptr && (lbhead == 0 || !p.lb_exact);
	const bool lbwarp = p.ok && p.lane_bases != nullptr && !lbtma;
	const uint32_t lbbytes = lbhead ? 144u : 128u;
	if (lbwarp) {
		for (uint32_t i = lane; i < 128; i += 32) { lbstage[lbhead + i] = p.lane_bases[i]; }
	}
	const bool tma_pk  = p.ok && p.bytes > 0 && (reinterpret_cast<uintptr_t>(p.src) & 15u) == 0;
	uint32_t   gwindow = 0;
	if (GSTAGE > 0 && p.ok && p.gbytes > 0) { gwindow = (p.ghead + p.gbytes + 15u) & ~15u; }
	if (GSTAGE > 0 && gwindow > GSTAGE) { gwindow = 0; }
	if (p.ok && p.bytes > 0 && !tma_pk) {
		if ((reinterpret_cast<uintptr_t>(p.src) & 3u) == 0) {
			const uint32_t* s = reinterpret_cast<const uint32_t*>(p.src);
			uint32_t*       d = reinterpret_cast<uint32_t*>(stage);
			for (uint32_t i = lane; i < p.bytes / 4; i += 32) { d[i] = s[i]; }
		} else {
			for (uint32_t i = lane; i < p.bytes; i += 32) { stage[i] = p.src[i]; }
		}
	}
	__syncwarp();
	if (lane == 0) {
		if (tma_pk) { tx += p.bytes; }
		tx += gwindow;
		if (lbtma) { tx += lbbytes; }
		mbar_arrive_expect_tx(bar, tx);
		// stall (failure injection): the byte count is armed, no copy is issued, so the wait runs out
		if (tma_pk && !stall) { bulk_g2s(stage, p.src, p.bytes, bar); }
		if (gwindow && !stall) { bulk_g2s(gstage, p.gsrc - p.ghead, gwindow, bar); }
		if (lbtma && !stall) { bulk_g2s(lbstage, p.lane_bases - lbhead, lbbytes, bar); }
		// without a staging area the run values are gathered from global memory: start them towards L2 now
		if (GSTAGE == 0 && p.ok && p.gbytes > 0) { bulk_prefetch_l2(p.gsrc - p.ghead, (p.ghead + p.gbytes + 15u) & ~15u); }
	}
}

#endif // FLS_HOST_EMULATION

// ---------------------------------------------------------------------------------------------------------
// Per-width decode of the staged stream into registers (run order).
// ---------------------------------------------------------------------------------------------------------
template <int WS>
struct StreamT {
	using T = uint32_t;
};
template <>
struct StreamT<64> {
	using T = uint64_t;
};

// Patch one vector's unpacked values (after the FOR add, before rsum) through `scratch` (1024 values in
// transposed order; the stage the packed words came from, free once they are in registers).  Exceptions are
// at p.gsrc (p.gbytes bytes), their positions / bitmap / chain head at p.dict (p.entry_c bytes).
template <int WS>
__device__ __forceinline__ void apply_patch(const Plan& p, typename StreamT<WS>::T (&v)[32], uint8_t* scratch,
                                            uint32_t t, int* status) {
	using T = typename StreamT<WS>::T;
	if constexpr (WS == 32 || WS == 64) {
		T*             s   = reinterpret_cast<T*>(scratch);
		const uint32_t n_e = p.gbytes / sizeof(T);
		__syncwarp();
#pragma unroll
		for (int q = 0; q < 32; ++q) { s[run_tpos<WS>(t, 0, q)] = v[q]; }
		__syncwarp();
		bool bad = false;
		if (p.post == POST_PATCH_S) {
			const uint32_t c = p.entry_c >= 2 ? static_cast<uint32_t>(ld_le(p.dict, 2)) : 0u;
			bad              = p.entry_c < 2 || 2u + 2u * c > p.entry_c || c > n_e;
			for (uint32_t i = t; !bad && i < c; i += 32) {
				const uint32_t pos = static_cast<uint32_t>(ld_le(p.dict + 2 + 2 * i, 2));
				if (pos < kVec) { s[pos] = static_cast<T>(ld_le(p.gsrc + static_cast<uint64_t>(i) * sizeof(T), sizeof(T))); }
			}
		} else if (p.post == POST_PATCH_B) {
			// 16 bitmap words, one per lane 0..15; exceptions follow the set bits in ascending order
			bad              = p.entry_c < 128;
			const uint64_t w = (!bad && t < 16) ? ld_le(p.dict + 8 * t, 8) : 0ull;
			const uint32_t c   = static_cast<uint32_t>(__popcll(w));
			uint32_t       inc = c; // inclusive warp scan of the per-word counts
#pragma unroll
			for (uint32_t d = 1; d < 32; d <<= 1) {
				const uint32_t y = __shfl_up_sync(0xFFFFFFFFu, inc, d);
				if (t >= d) { inc += y; }
			}
			const uint32_t i0  = inc - c;
			const uint32_t tot = __shfl_sync(0xFFFFFFFFu, inc, 31);
			bad |= tot > n_e;
			uint64_t rest = bad ? 0ull : w;
			for (uint32_t k = 0; rest != 0; ++k) {
				const uint32_t r = __ffsll(static_cast<long long>(rest)) - 1;
				rest &= rest - 1;
				s[64 * t + r] = static_cast<T>(ld_le(p.gsrc + static_cast<uint64_t>(i0 + k) * sizeof(T), sizeof(T)));
			}
		} else if (t == 0) {
			// LL: the packed value at an exception is the distance to the next one minus one
			const uint32_t c     = p.entry_c >= 4 ? static_cast<uint32_t>(ld_le(p.dict, 2)) : 0u;
			uint64_t       cur   = p.entry_c >= 4 ? ld_le(p.dict + 2, 2) : 0u;
			const T        base  = static_cast<T>(p.for_base);
			bad                  = p.entry_c < 4 || c > n_e;
			for (uint32_t i = 0; !bad && i < c; ++i) {
				if (cur >= kVec) {
					bad = true;
					break;
				}
				const T off = static_cast<T>(s[cur] - base + T(1));
				s[cur]      = static_cast<T>(ld_le(p.gsrc + static_cast<uint64_t>(i) * sizeof(T), sizeof(T)));
				cur += static_cast<uint64_t>(off);
			}
		}
		if (__any_sync(0xFFFFFFFFu, bad) && t == 0) { atomicOr(status, STATUS_BAD_INDEX); }
		__syncwarp();
#pragma unroll
		for (int q = 0; q < 32; ++q) { v[q] = s[run_tpos<WS>(t, 0, q)]; }
		__syncwarp();
	}
}

// The 32 values of half-lane h of lane l (values 2m + h, m = 0..31, in run order) of a 64-bit stream of bit
// width BW <= 16, as 32-bit words.  The thread's values sit at bits h*BW + 2m*BW of the lane: the lane's
// 32-bit words are first shifted by h*BW (one funnel shift each, every word read once), after which every
// value's word and shift are compile-time constants.
template <uint32_t BW>
__device__ __forceinline__ void extract_w64_small_bw(const uint32_t* __restrict__ S, uint32_t l, uint32_t h,
                                                     uint32_t (&x)[32]) {
	constexpr uint32_t mask = BW == 0 ? 0u : (1u << BW) - 1u;
	if constexpr (BW == 0) {
#pragma unroll
		for (int i = 0; i < 32; ++i) { x[i] = 0; }
	} else {
		const uint32_t hb  = h * BW;
		// lane word k (k = 0, 1, ...: the low and high halves of the lane's 64-bit words in order)
		auto           raw = [&](uint32_t k) { return S[2 * (l + 16 * (k >> 1)) + (k & 1u)]; };
#pragma unroll
		for (uint32_t m = 0; m < 32; ++m) {
			const uint32_t b  = 2 * m * BW;
			const uint32_t k  = b >> 5;
			const uint32_t sh = b & 31u;
			const uint32_t s0 = __funnelshift_r(raw(k), raw(k + 1), hb);
			if (sh + BW <= 32) {
				x[run32_pos(m)] = (s0 >> sh) & mask;
			} else {
				const uint32_t s1 = __funnelshift_r(raw(k + 1), raw(k + 2), hb);
				x[run32_pos(m)]   = __funnelshift_r(s0, s1, sh) & mask;
			}
		}
	}
}

// Bit widths up to 26 (values below 2^26): compile-time layouts up to 16 bits, computed offsets above.
__device__ __forceinline__ void extract_w64_small(const uint32_t* __restrict__ S, uint32_t l, uint32_t h,
                                                  uint32_t bw, uint32_t (&x)[32]) {
	switch (bw) {
#define FLS_W64_SMALL(B)                                                                                               \
	case B: extract_w64_small_bw<B>(S, l, h, x); return;
		FLS_W64_SMALL(0) FLS_W64_SMALL(1) FLS_W64_SMALL(2) FLS_W64_SMALL(3) FLS_W64_SMALL(4) FLS_W64_SMALL(5)
		FLS_W64_SMALL(6) FLS_W64_SMALL(7) FLS_W64_SMALL(8) FLS_W64_SMALL(9) FLS_W64_SMALL(10) FLS_W64_SMALL(11)
		FLS_W64_SMALL(12) FLS_W64_SMALL(13) FLS_W64_SMALL(14) FLS_W64_SMALL(15) FLS_W64_SMALL(16)
#undef FLS_W64_SMALL
	default: break;
	}
	const uint32_t mlo = (1u << bw) - 1u;
#pragma unroll
	for (uint32_t m = 0; m < 32; ++m) {
		const uint32_t b  = (2 * m + h) * bw;
		const uint32_t h2 = b >> 5;
		const uint32_t lo = S[2 * (l + 16 * (h2 >> 1)) + (h2 & 1u)];
		const uint32_t h3 = h2 + 1;
		const uint32_t hi = S[2 * (l + 16 * (h3 >> 1)) + (h3 & 1u)];
		x[run32_pos(m)]   = __funnelshift_r(lo, hi, b & 31u) & mlo;
	}
}

// PATCH: the kernel may meet patched items (plain-stream kernels and the catch-all one; gather kernels never do)
template <int WS, bool PATCH = true>
__device__ __forceinline__ void decode_stream(const Plan& p, const uint32_t* S, uint32_t t,
                                              typename StreamT<WS>::T (&v)[32], uint8_t* scratch = nullptr,
                                              int* status = nullptr) {
	using T = typename StreamT<WS>::T;
	if constexpr (WS == 64) {
		if (p.enc == ENC_DELTA && p.bw <= 26 && p.for_base < (1ull << 26) &&
		    !(PATCH && scratch && post_is_patch(p.post))) {
			// small deltas (the common case of sorted 64-bit keys): every delta + FOR base is below 2^27, so a
			// half-lane's running sum of 32 of them fits 32 bits; the 64-bit add happens once per value
			const uint32_t l   = t & 15u;
			const uint32_t h   = t >> 4;
			const uint32_t b32 = static_cast<uint32_t>(p.for_base);
			uint32_t       x[32];
			extract_w64_small(S, l, h, p.bw, x);
			uint32_t acc = 0;
#pragma unroll
			for (int i = 0; i < 32; ++i) {
				acc += x[i] + b32;
				x[i] = acc;
			}
			const uint32_t lower = __shfl_sync(0xFFFFFFFFu, acc, l); // total of the lane's first half
			const T        add   = static_cast<T>(ld_le(p.lane_bases + 8 * l, 8)) + (h ? lower : 0u);
#pragma unroll
			for (int i = 0; i < 32; ++i) { v[i] = add + x[i]; }
			return;
		}
		extract_w64(S, t, p.bw, v);
	} else if constexpr (WS == 32) {
		extract_w32(S, t, p.bw, v);
	} else if constexpr (WS == 16) {
		extract_w16(S, t, p.bw, v);
	} else {
		extract_w8(S, t, p.bw, v);
	}
	constexpr T wmask = WS == 64 ? ~T(0) : static_cast<T>((1ull << WS) - 1ull);
	// 16- and 8-bit DELTA streams without patches add the FOR base inside the running sum: sums of at most 16
	// terms below 2^16 stay exact in 32 bits, so the wrap to the stream width comes once per value, off the
	// chain of dependent adds
	const bool fold = WS <= 16 && p.enc == ENC_DELTA && !(PATCH && scratch && post_is_patch(p.post));
	if (p.enc != ENC_RAW && !fold) {
		const T base = static_cast<T>(p.for_base);
#pragma unroll
		for (int i = 0; i < 32; ++i) { v[i] = (v[i] + base) & wmask; }
	}
	if constexpr (PATCH) {
		if (scratch && post_is_patch(p.post)) { apply_patch<WS>(p, v, scratch, t, status); }
	}
	if (p.enc == ENC_DELTA) {
		// rsum: running sum along each lane in original order, seeded by the lane's base.
		if constexpr (WS == 32) {
			T acc = static_cast<T>(ld_le(p.lane_bases + 4 * t, 4));
#pragma unroll
			for (int i = 0; i < 32; ++i) {
				acc += v[i];
				v[i] = acc;
			}
		} else if constexpr (WS == 64) {
			const uint32_t l   = t & 15u;
			const uint32_t h   = t >> 4;
			T              acc = 0;
#pragma unroll
			for (int i = 0; i < 32; ++i) {
				acc += v[i];
				v[i] = acc;
			}
			const T lower = __shfl_sync(0xFFFFFFFFu, acc, l); // total of the lane's first half
			T       add   = static_cast<T>(ld_le(p.lane_bases + 8 * l, 8));
			if (h) { add += lower; }
#pragma unroll
			for (int i = 0; i < 32; ++i) { v[i] += add; }
		} else if constexpr (WS == 16) {
			const T base = fold ? static_cast<T>(p.for_base) & wmask : T(0);
#pragma unroll
			for (int q = 0; q < 2; ++q) {
				T acc = static_cast<T>(ld_le(p.lane_bases + 2 * (2 * t + q), 2));
#pragma unroll
				for (int i = 0; i < 16; ++i) {
					acc += v[16 * q + i] + base;
					v[16 * q + i] = acc;
				}
			}
#pragma unroll
			for (int i = 0; i < 32; ++i) { v[i] &= wmask; }
		} else {
			const T base = fold ? static_cast<T>(p.for_base) & wmask : T(0);
#pragma unroll
			for (int q = 0; q < 4; ++q) {
				T acc = p.lane_bases[4 * t + q];
#pragma unroll
				for (int i = 0; i < 8; ++i) {
					acc += v[8 * q + i] + base;
					v[8 * q + i] = acc;
				}
			}
#pragma unroll
			for (int i = 0; i < 32; ++i) { v[i] &= wmask; }
		}
	}
}

// ---------------------------------------------------------------------------------------------------------
// Store of 32 values per thread (run order) for stream width WS and element size E.
// ---------------------------------------------------------------------------------------------------------
template <int E>
struct OutT {
	using T = uint32_t;
};
template <>
struct OutT<8> {
	using T = uint64_t;
};
// exact element type of an E-byte output
template <int E>
struct ElemT;
template <>
struct ElemT<1> {
	using T = uint8_t;
};
template <>
struct ElemT<2> {
	using T = uint16_t;
};
template <>
struct ElemT<4> {
	using T = uint32_t;
};
template <>
struct ElemT<8> {
	using T = uint64_t;
};

template <int WS, int E>
__device__ __forceinline__ void store_vector(const typename OutT<E>::T (&o)[32], uint8_t* out, uint8_t* ost,
                                             bool original, uint32_t t) {
	constexpr uint32_t RL = run_len<WS>();
	constexpr uint32_t RC = run_count<WS>();
	if (original) {
		__syncwarp(); // the staging buffer is the stage the packed words were just read from
#pragma unroll
		for (uint32_t r = 0; r < RC; ++r) {
			const uint32_t b0 = run_start<WS>(t, r) * E;
			if constexpr (RL * E >= 16) {
				constexpr uint32_t PER = 16 / E; // values per 16-byte chunk
#pragma unroll
				for (uint32_t c = 0; c < RL * E / 16; ++c) {
					uint32_t w[4];
#pragma unroll
					for (uint32_t k = 0; k < 4; ++k) {
						if constexpr (E == 8) {
							const uint64_t x = o[r * RL + c * PER + k / 2];
							w[k]             = (k & 1) ? static_cast<uint32_t>(x >> 32) : static_cast<uint32_t>(x);
						} else if constexpr (E == 4) {
							w[k] = static_cast<uint32_t>(o[r * RL + c * PER + k]);
						} else if constexpr (E == 2) {
							w[k] = (o[r * RL + c * PER + 2 * k] & 0xFFFFu) | (o[r * RL + c * PER + 2 * k + 1] << 16);
						} else {
							const uint32_t i0 = r * RL + c * PER + 4 * k;
							w[k] = (o[i0] & 0xFFu) | ((o[i0 + 1] & 0xFFu) << 8) | ((o[i0 + 2] & 0xFFu) << 16) |
							       (o[i0 + 3] << 24);
						}
					}
					*reinterpret_cast<uint4*>(ost + stage_off(b0 + 16 * c)) = make_uint4(w[0], w[1], w[2], w[3]);
				}
			} else {
				// WS = 8, E = 1: an 8-byte run
				const uint32_t i0 = r * RL;
				const uint32_t lo = (o[i0] & 0xFFu) | ((o[i0 + 1] & 0xFFu) << 8) | ((o[i0 + 2] & 0xFFu) << 16) |
				                    (o[i0 + 3] << 24);
				const uint32_t hi = (o[i0 + 4] & 0xFFu) | ((o[i0 + 5] & 0xFFu) << 8) |
				                    ((o[i0 + 6] & 0xFFu) << 16) | (o[i0 + 7] << 24);
				*reinterpret_cast<uint2*>(ost + stage_off(b0)) = make_uint2(lo, hi);
			}
		}
		__syncwarp();
		if ((reinterpret_cast<uintptr_t>(out) & 15u) == 0) {
#pragma unroll
			for (uint32_t c = t; c < 64u * E; c += 32) {
				const uint4 x = *reinterpret_cast<const uint4*>(ost + stage_off(16 * c));
				*reinterpret_cast<uint4*>(out + 16 * c) = x;
			}
		} else {
			for (uint32_t b = t; b < 1024u * E; b += 32) { out[b] = ost[stage_off(b)]; }
		}
		__syncwarp();
	} else {
		using ET = typename ElemT<E>::T;
#pragma unroll
		for (uint32_t p = 0; p < RL; ++p) {
			// the thread's RC lanes are adjacent in the transposed order
			const uint32_t k0 = run_tpos<WS>(t, 0, p);
#pragma unroll
			for (uint32_t r = 0; r < RC; ++r) { reinterpret_cast<ET*>(out)[k0 + r] = static_cast<ET>(o[r * RL + p]); }
		}
	}
}

// ---------------------------------------------------------------------------------------------------------
// Predicate of 32 values per thread (run order) into the vector's 1024-bit bitmap at out (predicate pushdown:
// the decoded values never leave the registers).  Bit i of the bitmap is value i of the vector in the plan's
// order (original or transposed).
// ---------------------------------------------------------------------------------------------------------
// The predicate for E-byte values: the classes (below / equal / above the constant) it accepts, and the
// constant in the values' own width when it lies inside their range (else every value is in one class).
template <int E>
struct PredE {
	using T = typename OutT<E>::T;
	uint32_t accept; // bit 0: value < constant, bit 1: ==, bit 2: >
	uint32_t fixed;  // 0: compare; else the class bit of every value (constant outside the values' range)
	bool     sgn;
	T        c;

	__device__ __forceinline__ PredE(const Pred& pr, bool is_signed) : sgn(is_signed) {
		// accepted classes of EQ NE LT LE GT GE: 2, 5, 1, 3, 4, 6 (one nibble each)
		accept = (0x643152u >> (4 * (pr.op < 6 ? pr.op : 0))) & 7u;
		fixed  = 0;
		if constexpr (E == 8) {
			c = pr.value;
		} else {
			const int64_t v = static_cast<int64_t>(pr.value);
			if (sgn) {
				const int64_t lo = -(1ll << (8 * E - 1)), hi = (1ll << (8 * E - 1)) - 1;
				fixed            = v < lo ? 4u : v > hi ? 1u : 0u; // below the range: every value is above it
			} else {
				const uint64_t hi = (1ull << (8 * E)) - 1;
				fixed             = pr.value > hi ? 1u : 0u;
			}
			c = static_cast<T>(pr.value);
		}
	}
	// class bit of x: 1 below, 2 equal, 4 above the constant
	__device__ __forceinline__ uint32_t cls(T x) const {
		if constexpr (E == 8) {
			const bool lt = sgn ? static_cast<int64_t>(x) < static_cast<int64_t>(c) : x < c;
			return x == c ? 2u : lt ? 1u : 4u;
		} else {
			if (fixed) { return fixed; }
			constexpr uint32_t sh = 32 - 8 * E;
			const uint32_t     xu = static_cast<uint32_t>(x) << sh; // the value's E bytes at the top
			const uint32_t     cu = static_cast<uint32_t>(c) << sh;
			const bool lt = sgn ? static_cast<int32_t>(xu) < static_cast<int32_t>(cu) : xu < cu;
			return xu == cu ? 2u : lt ? 1u : 4u;
		}
	}
	__device__ __forceinline__ bool operator()(T x) const { return (cls(x) & accept) != 0; }
};

// 16 bits to the even bits of a word
__device__ __forceinline__ uint32_t spread16(uint32_t x) {
	x = (x | (x << 8)) & 0x00FF00FFu;
	x = (x | (x << 4)) & 0x0F0F0F0Fu;
	x = (x | (x << 2)) & 0x33333333u;
	return (x | (x << 1)) & 0x55555555u;
}

template <int WS, int E>
__device__ __forceinline__ void filter_vector(const typename OutT<E>::T (&o)[32], const Plan& p, uint8_t* ost,
                                              uint32_t t, const Pred& pr) {
	constexpr uint32_t RL = run_len<WS>();
	constexpr uint32_t RC = run_count<WS>();
	const PredE<E>     holds(pr, p.cmp == OUT_BITMAP_S);
	uint32_t*          out  = reinterpret_cast<uint32_t*>(p.out);
	uint32_t           mine = 0; // bitmap word t
	if (p.order) {
		if constexpr (RL == 32) {
			// the thread's run is one aligned bitmap word
#pragma unroll
			for (uint32_t j = 0; j < 32; ++j) { mine |= static_cast<uint32_t>(holds(o[j])) << j; }
			out[run_start<WS>(t, 0) / 32] = mine;
			return;
		} else {
			// runs of RL (16 or 8) values start at multiples of 8: every bitmap byte belongs to one run
			__syncwarp(); // the stage was just read into registers
#pragma unroll
			for (uint32_t r = 0; r < RC; ++r) {
				uint32_t m = 0;
#pragma unroll
				for (uint32_t j = 0; j < RL; ++j) { m |= static_cast<uint32_t>(holds(o[r * RL + j])) << j; }
				const uint32_t s = run_start<WS>(t, r) / 8;
#pragma unroll
				for (uint32_t b = 0; b < RL / 8; ++b) { ost[s + b] = static_cast<uint8_t>(m >> (8 * b)); }
			}
			__syncwarp();
			mine = reinterpret_cast<const uint32_t*>(ost)[t];
		}
	} else if constexpr (WS == 32 || WS == 64) {
		// run position j of every thread lands on bit t of bitmap word run32_val(j)
#pragma unroll
		for (uint32_t j = 0; j < 32; ++j) {
			const uint32_t b = __ballot_sync(0xFFFFFFFFu, holds(o[j]));
			if (run32_val(j) == t) { mine = b; }
		}
	} else if constexpr (WS == 16) {
		// run position j of the thread's two lanes: bits 2t and 2t + 1 of the 64 at 64 * run16_val(j)
#pragma unroll
		for (uint32_t j = 0; j < 16; ++j) {
			const uint32_t b0 = __ballot_sync(0xFFFFFFFFu, holds(o[j]));
			const uint32_t b1 = __ballot_sync(0xFFFFFFFFu, holds(o[16 + j]));
			const uint32_t g  = 2 * run16_val(j);
			if (t == g) { mine = spread16(b0 & 0xFFFFu) | (spread16(b1 & 0xFFFFu) << 1); }
			if (t == g + 1) { mine = spread16(b0 >> 16) | (spread16(b1 >> 16) << 1); }
		}
	} else {
		uint32_t* bm = reinterpret_cast<uint32_t*>(ost);
		__syncwarp();
		bm[t] = 0;
		__syncwarp();
#pragma unroll
		for (uint32_t r = 0; r < RC; ++r) {
#pragma unroll
			for (uint32_t j = 0; j < RL; ++j) {
				if (holds(o[r * RL + j])) {
					const uint32_t k = run_tpos<WS>(t, r, j);
					atomicOr(bm + k / 32, 1u << (k & 31u));
				}
			}
		}
		__syncwarp();
		mine = bm[t];
	}
	out[t] = mine;
	__syncwarp();
}

// ---------------------------------------------------------------------------------------------------------
// Full decode of one staged vector.
// ---------------------------------------------------------------------------------------------------------
// GSMEM: RLE run values / run codes staged in shared memory at gstage + ghead (else read from p.gsrc).
// KIND: bit 0 = the kernel handles RLE / DICT gathers, bit 1 = patched FFOR / DELTA items; a kernel that meets
// an item outside its kind flags a layout error (plans never route one there).  Bit 2 (KIND_FILTER): the
// vector's predicate bitmap is written instead of its values.
enum : int { KIND_PLAIN = 0, KIND_GATHER = 1, KIND_PATCH = 2, KIND_ALL = 3, KIND_FILTER = 4 };

template <int WS, int E, bool GSMEM = true, int KIND = KIND_ALL>
__device__ __forceinline__ void decode_vector(const Plan& p, const uint8_t* stage, const uint8_t* gstage, uint8_t* ost,
                                              uint32_t t, int* status, const Pred& pr = Pred {}) {
	using ST = typename StreamT<WS>::T;
	using OT = typename OutT<E>::T;
	ST v[32];
	constexpr bool GATHER = (KIND & KIND_GATHER) != 0;
	constexpr bool PATCH  = (KIND & KIND_PATCH) != 0;
	decode_stream<WS, PATCH>(p, reinterpret_cast<const uint32_t*>(stage), t, v, ost, status);
	if (!PATCH && post_is_patch(p.post) && t == 0) { atomicOr(status, STATUS_BAD_LAYOUT); }
	OT o[32];
	bool bad = false;
	if (!GATHER || !post_is_gather(p.post)) {
#pragma unroll
		for (int i = 0; i < 32; ++i) { o[i] = static_cast<OT>(v[i]); }
		if (!GATHER && post_is_gather(p.post) && t == 0) { atomicOr(status, STATUS_BAD_LAYOUT); }
	} else if (p.post == POST_RLE) {
		// run values keep the byte alignment they have inside the page
		const uint8_t* vals = GSMEM ? gstage + p.ghead : p.gsrc;
		if (!GSMEM && (reinterpret_cast<uintptr_t>(vals) & (E - 1)) == 0) {
			// naturally aligned run values (the usual case): plain loads, no per-value alignment test
			using VT        = typename ElemT<E>::T;
			const VT* tvals = reinterpret_cast<const VT*>(vals);
#pragma unroll
			for (int i = 0; i < 32; ++i) {
				const uint32_t idx = static_cast<uint32_t>(v[i]);
				const bool     in  = idx < p.n_runs;
				bad |= !in;
				o[i] = in ? static_cast<OT>(tvals[idx]) : OT(0);
			}
		} else {
#pragma unroll
			for (int i = 0; i < 32; ++i) {
				const uint32_t idx = static_cast<uint32_t>(v[i]);
				const bool     in  = idx < p.n_runs;
				bad |= !in;
				const uint8_t* a = vals + static_cast<uint64_t>(idx) * E;
				o[i] = !in ? OT(0) : GSMEM ? static_cast<OT>(sld<E>(a)) : static_cast<OT>(ld_le(a, E));
			}
		}
	} else {
		const uint8_t* codes        = GSMEM ? gstage + p.ghead : p.gsrc;
		const bool     dict_aligned = (reinterpret_cast<uintptr_t>(p.dict) & (E - 1)) == 0;
#pragma unroll
		for (int i = 0; i < 32; ++i) {
			uint32_t code = static_cast<uint32_t>(v[i]);
			if (p.post == POST_RLE_DICT) {
				const bool     in = code < p.n_runs;
				const uint8_t* a  = codes + 4ull * code;
				bad |= !in;
				code = !in ? 0u : GSMEM ? sld4(a) : static_cast<uint32_t>(ld_le(a, 4));
			}
			const bool in = code < p.entry_c;
			bad |= !in;
			const uint8_t* a = p.dict + static_cast<uint64_t>(code) * E;
			o[i] = !in ? OT(0) : dict_aligned ? static_cast<OT>(*reinterpret_cast<const typename ElemT<E>::T*>(a))
			                                  : static_cast<OT>(ld_le(a, E));
		}
	}
	if (__any_sync(0xFFFFFFFFu, bad) && t == 0) { atomicOr(status, STATUS_BAD_INDEX); }
	if constexpr ((KIND & KIND_FILTER) != 0) {
		bool values = false;
		if constexpr ((KIND & KIND_PATCH) != 0) {
			// an intermediate stream of a filter plan (a DICT page's patched codes, a patched item)
			values = p.cmp == OUT_VALUES;
			if (values) { store_vector<WS, E>(o, p.out, ost, p.order != 0, t); }
		}
		if (!values) { filter_vector<WS, E>(o, p, ost, t, pr); }
	} else {
		store_vector<WS, E>(o, p.out, ost, p.order != 0, t);
	}
}

// Compact plan kept in shared memory between the lane-parallel metadata fetch and the use of the plan.
struct __align__(16) PlanS {
	const uint8_t* src;
	uint8_t*       out;
	uint64_t       for_base;
	const uint8_t* lane_bases;
	const uint8_t* gsrc;
	const uint8_t* dict;
	uint32_t       gbytes;
	uint32_t       entry_c;
	uint16_t       bytes;
	uint8_t        bw, ws, e, enc, post, flags; // flags: bit0 original order, bit1 ok, bit2 valid, bit3 lb_exact,
	                                            // bits 4-5 cmp
};
static_assert(sizeof(PlanS) == 64, "PlanS layout");

__device__ __forceinline__ PlanS pack_plan(const Plan& p, bool valid) {
	PlanS s;
	s.src        = p.src;
	s.out        = p.out;
	s.for_base   = p.for_base;
	s.lane_bases = p.lane_bases;
	s.gsrc       = p.gsrc;
	s.dict       = p.dict;
	s.gbytes     = p.gbytes;
	s.entry_c    = p.entry_c;
	s.bytes      = static_cast<uint16_t>(p.bytes);
	s.bw         = static_cast<uint8_t>(p.bw > 255 ? 255 : p.bw);
	s.ws         = p.ws;
	s.e          = p.e;
	s.enc        = p.enc;
	s.post       = p.post;
	s.flags      = static_cast<uint8_t>((p.order ? 1 : 0) | (p.ok ? 2 : 0) | (valid ? 4 : 0) | (p.lb_exact ? 8 : 0) |
	                                    ((p.cmp & 3u) << 4));
	return s;
}

__device__ __forceinline__ Plan unpack_plan(const PlanS& s) {
	Plan p;
	p.src        = s.src;
	p.out        = s.out;
	p.for_base   = s.for_base;
	p.lane_bases = s.lane_bases;
	p.gsrc       = s.gsrc;
	p.dict       = s.dict;
	p.gbytes     = s.gbytes;
	p.entry_c    = s.entry_c;
	p.bytes      = s.bytes;
	p.bw         = s.bw;
	p.ws         = s.ws;
	p.e          = s.e;
	p.enc        = s.enc;
	p.post       = s.post;
	p.order      = s.flags & 1u;
	p.ok         = (s.flags & 2u) != 0;
	p.lb_exact   = (s.flags & 8u) != 0;
	p.cmp        = (s.flags >> 4) & 3u;
	const uint32_t ve = p.post == POST_RLE ? p.e : 4u;
	p.n_runs     = (p.post == POST_RLE || p.post == POST_RLE_DICT) ? p.gbytes / ve : 0u;
	p.ghead      = static_cast<uint32_t>(reinterpret_cast<uintptr_t>(p.gsrc) & 15u);
	return p;
}

#ifndef FLS_HOST_EMULATION
__device__ __forceinline__ uint32_t item_col(uint32_t it, uint32_t shift) { return it >> shift; }
__device__ __forceinline__ uint32_t item_vec(uint32_t it, uint32_t shift) { return it & ((1u << shift) - 1u); }

__device__ __forceinline__ Plan plan_of(const DecodeArgs& a, uint64_t item) {
	if (a.queue == nullptr) { return make_plan(a.col0, static_cast<uint32_t>(item)); }
	const uint32_t it = a.queue[item];
	const ColDesc& c  = a.cols ? a.cols[item_col(it, a.col_shift)] : a.col0;
	return make_plan(c, item_vec(it, a.col_shift));
}

// Kernel family: MAXWS bounds the staged stream (MAXWS * 128 bytes), GSTAGE the run-value window, EMAX the
// output element size.  The original-order staging reuses the stage once its packed words are in registers,
// so a slot is max(stream, output) bytes plus the run-value window.  Plans of the warp's next 2*PB items
// live in shared memory (64 bytes each).
template <int MAXWS, uint32_t GSTAGE, int EMAX, int WARPS, int STAGES, int KIND = KIND_ALL>
struct Geometry {
	static constexpr uint32_t kPB      = 16;
	static constexpr uint32_t kStage   = MAXWS * 128u;
	static constexpr uint32_t kOut     = EMAX * 1024u;
	static constexpr uint32_t kMain    = kStage > kOut ? kStage : kOut;
	static constexpr uint32_t kSlot    = kMain + kLaneWindow + GSTAGE;
	static constexpr uint32_t kPlans   = 2 * kPB * sizeof(PlanS);
	static constexpr uint32_t kPerWarp = 64u + kPlans + STAGES * kSlot;
	static constexpr uint32_t kSlack   = 256u; // extraction reads one row past the last stage
	static constexpr uint32_t kSmem    = WARPS * kPerWarp + kSlack;
	static constexpr int      kThreads = WARPS * 32;
	static_assert(STAGES < kPB, "plans must run ahead of the copies");
	static_assert(kSmem <= 232448u, "at most 227 KB of shared memory per CTA");
};

template <int MAXWS, uint32_t GSTAGE, int EMAX, int KIND>
__device__ __forceinline__ void decode_dispatch(const Plan& p, uint8_t* st, const uint8_t* gs, uint32_t lane,
                                                int* status, const Pred& pr) {
	if (p.ws == 64) {
		if constexpr (MAXWS >= 64) { decode_vector<64, 8, (GSTAGE > 0), KIND>(p, st, gs, st, lane, status, pr); }
	} else if (p.ws == 32) {
		if constexpr (MAXWS >= 32) {
			if (p.e == 8) {
				if constexpr (EMAX >= 8) { decode_vector<32, 8, (GSTAGE > 0), KIND>(p, st, gs, st, lane, status, pr); }
			} else {
				decode_vector<32, 4, (GSTAGE > 0), KIND>(p, st, gs, st, lane, status, pr);
			}
		}
	} else if (p.ws == 16) {
		if (p.e == 8) {
			if constexpr (EMAX >= 8) { decode_vector<16, 8, (GSTAGE > 0), KIND>(p, st, gs, st, lane, status, pr); }
		} else if (p.e == 4) {
			if constexpr (EMAX >= 4) { decode_vector<16, 4, (GSTAGE > 0), KIND>(p, st, gs, st, lane, status, pr); }
		} else {
			decode_vector<16, 2, (GSTAGE > 0), KIND>(p, st, gs, st, lane, status, pr);
		}
	} else {
		decode_vector<8, 1, (GSTAGE > 0), KIND>(p, st, gs, st, lane, status, pr);
	}
}

template <int MAXWS, uint32_t GSTAGE, int EMAX, int WARPS, int STAGES, int KIND>
__global__ void __launch_bounds__(WARPS * 32, 1) k_decode(const DecodeArgs a) {
	using G = Geometry<MAXWS, GSTAGE, EMAX, WARPS, STAGES, KIND>;
	constexpr uint32_t PB = G::kPB;
	extern __shared__ __align__(128) uint8_t smem[];
	const uint32_t lane   = threadIdx.x & 31u;
	const uint32_t warp   = threadIdx.x >> 5;
	uint8_t*       wbase  = smem + warp * G::kPerWarp;
	uint64_t*      bars   = reinterpret_cast<uint64_t*>(wbase);
	PlanS*         plans  = reinterpret_cast<PlanS*>(wbase + 64);
	uint8_t*       stages = wbase + 64 + G::kPlans;

	if (lane == 0) {
		for (int s = 0; s < STAGES; ++s) { mbar_init(&bars[s], 1); }
		fence_mbar_init();
	}

	const uint64_t gw = static_cast<uint64_t>(blockIdx.x) * WARPS + warp;
	const uint64_t nw = static_cast<uint64_t>(gridDim.x) * WARPS;
	const uint64_t n  = a.n_items;

	auto stage_ptr  = [&](uint32_t s) { return stages + s * G::kSlot; };
	auto lb_ptr     = [&](uint32_t s) { return stages + s * G::kSlot + G::kMain; };
	auto gstage_ptr = [&](uint32_t s) { return stages + s * G::kSlot + G::kMain + kLaneWindow; };
	// Lane-parallel metadata fetch: lane j resolves the plan of the warp's item blk*PB + j.
	auto fill = [&](uint32_t blk) {
		if (lane < PB) {
			const uint64_t k    = static_cast<uint64_t>(blk) * PB + lane;
			const uint64_t item = gw + k * nw;
			Plan           p {};
			const bool     valid = item < n;
			if (valid) { p = plan_of(a, item); }
			plans[k % (2 * PB)] = pack_plan(p, valid);
		}
	};
	auto issue_k = [&](uint64_t k, uint32_t s) {
		const PlanS& ps = plans[k % (2 * PB)];
		if (ps.flags & 4u) {
			const bool stall = a.test_stall != 0 && gw + k * nw == a.test_stall - 1;
			issue<GSTAGE>(unpack_plan(ps), stage_ptr(s), gstage_ptr(s), lb_ptr(s), &bars[s], lane, stall);
		}
	};
	const uint32_t limit = a.spin_limit ? a.spin_limit : kMbarSpinLimit;

	fill(0);
	fill(1);
	__syncwarp();
	for (uint32_t s = 0; s < STAGES; ++s) { issue_k(s, s); }

	uint32_t k       = 0;
	bool     aborted = false;
	for (uint64_t item = gw; item < n; item += nw, ++k) {
		if (k % PB == 0 && k > 0) {
			fill(k / PB + 1);
			__syncwarp();
		}
		const uint32_t s      = k % STAGES;
		const uint32_t parity = (k / STAGES) & 1u;
		Plan           p      = unpack_plan(plans[k % (2 * PB)]);
		if (!mbar_wait(&bars[s], parity, limit)) {
			if (lane == 0) { atomicOr(a.status, STATUS_TIMEOUT); }
			aborted = true;
			break;
		}
		if (!p.ok) {
			if (lane == 0) { atomicOr(a.status, p.bw > p.ws ? STATUS_BAD_BW : STATUS_BAD_LAYOUT); }
		} else {
			// the lane bases were staged with the packed words
			if (p.lane_bases) { p.lane_bases = lb_ptr(s) + (reinterpret_cast<uintptr_t>(p.lane_bases) & 15u); }
			decode_dispatch<MAXWS, GSTAGE, EMAX, KIND>(p, stage_ptr(s), gstage_ptr(s), lane, a.status, a.pred);
		}
		__syncwarp();
		issue_k(k + STAGES, s);
	}
	if (aborted) {
		// Drain: every later stage this warp armed must land before the block's shared memory goes away (full
		// bound: these copies were issued)
		for (uint32_t j = k + 1; j < k + STAGES; ++j) {
			const uint64_t item = gw + static_cast<uint64_t>(j) * nw;
			if (item >= n) { break; }
			(void)mbar_wait(&bars[j % STAGES], (j / STAGES) & 1u);
		}
	}
}
#endif // FLS_HOST_EMULATION

} // namespace flsgpu
