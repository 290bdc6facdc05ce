// Warp emulation of the decode engine's device logic (fastlanes_b200/csrc/fls_decode.cu) on the CPU.
// make_plan / decode_vector run unchanged; one warp = 32 std::threads; "shared memory" is a host buffer the
// harness fills the way the kernel's bulk copies would.  Used by tests/test_device_logic_emulated.py.
#define FLS_HOST_EMULATION 1
#include "fls_decode.cu"
#include "fls_page.h"
#include "fls_strings.cuh"
#include "fls_b200.h"

#include <thread>
#include <vector>

thread_local EmuWarp* g_emu_warp = nullptr;
thread_local int      g_emu_lane = 0;

using namespace flsgpu;

template <int K = KIND_ALL>
static void dispatch(const Plan& p, const uint8_t* st, const uint8_t* gs, uint8_t* ost, uint32_t t, int* status,
                     const Pred& pr = Pred {}) {
	if (p.ws == 64) {
		decode_vector<64, 8, true, K>(p, st, gs, ost, t, status, pr);
	} else if (p.ws == 32) {
		if (p.e == 8) {
			decode_vector<32, 8, true, K>(p, st, gs, ost, t, status, pr);
		} else {
			decode_vector<32, 4, true, K>(p, st, gs, ost, t, status, pr);
		}
	} else if (p.ws == 16) {
		if (p.e == 8) {
			decode_vector<16, 8, true, K>(p, st, gs, ost, t, status, pr);
		} else if (p.e == 4) {
			decode_vector<16, 4, true, K>(p, st, gs, ost, t, status, pr);
		} else {
			decode_vector<16, 2, true, K>(p, st, gs, ost, t, status, pr);
		}
	} else {
		decode_vector<8, 1, true, K>(p, st, gs, ost, t, status, pr);
	}
}

static int emu_vector(const ColDesc& c, uint32_t v, const Pred* filter = nullptr) {
	Plan p = make_plan(c, v);
	if (!p.ok) { return p.bw > p.ws ? STATUS_BAD_BW : STATUS_BAD_LAYOUT; }
	std::vector<uint8_t> smem(3 * 8448 + 8192, 0xA5);
	uint8_t*             stage  = smem.data();
	uint8_t*             gstage = stage + 8448;
	if (p.bytes) { std::memcpy(stage, p.src, p.bytes); }
	if (p.gbytes) {
		const uint32_t win = (p.ghead + p.gbytes + 15u) & ~15u;
		std::memcpy(gstage, p.gsrc - p.ghead, win);
	}
	std::vector<uint8_t> lbwin(256 + 16, 0xA5);
	if (p.lane_bases) {
		// as on the GPU: the 16-byte aligned 144-byte window around the lane bases, staged
		uint8_t*        lb   = reinterpret_cast<uint8_t*>((reinterpret_cast<uintptr_t>(lbwin.data()) + 15) & ~uintptr_t(15));
		const uintptr_t head = reinterpret_cast<uintptr_t>(p.lane_bases) & 15u;
		if (p.lb_exact || head == 0) {
			std::memcpy(lb + head, p.lane_bases, 128);
		} else {
			std::memcpy(lb, p.lane_bases - head, 144);
		}
		p.lane_bases = lb + head;
	}
	int                      status = 0;
	std::barrier<>           bar(32);
	EmuWarp                  w {&bar, {}, {}};
	std::vector<std::thread> th;
	for (int t = 0; t < 32; ++t) {
		th.emplace_back([&, t] {
			g_emu_warp = &w;
			g_emu_lane = t;
			// as on the GPU: staging reuses the stage
			if (filter) {
				dispatch<KIND_ALL | KIND_FILTER>(p, stage, gstage, stage, static_cast<uint32_t>(t), &status, *filter);
			} else {
				dispatch(p, stage, gstage, stage, static_cast<uint32_t>(t), &status);
			}
		});
	}
	for (auto& x : th) { x.join(); }
	return status;
}

extern "C" int emu_decode_column(const ColDesc* c) {
	int st = 0;
	for (uint32_t v = 0; v < c->n_vec; ++v) { st |= emu_vector(*c, v); }
	return st;
}

extern "C" int emu_unffor(int width, int enc, int order, const uint8_t* packed, const uint64_t* byte_off,
                          const uint8_t* bw, const uint8_t* base, const uint8_t* lane_base, uint64_t n_vec,
                          uint8_t* out) {
	ColDesc c {};
	c.ws            = static_cast<uint8_t>(width);
	c.e             = static_cast<uint8_t>(width / 8);
	c.enc           = static_cast<uint8_t>(enc);
	c.post          = POST_NONE;
	c.order         = static_cast<uint8_t>(order);
	c.layout        = LAYOUT_ARRAYS;
	c.n_vec         = static_cast<uint32_t>(n_vec);
	c.bw_const      = enc == ENC_RAW ? static_cast<uint8_t>(width) : 0;
	c.packed        = packed;
	c.byte_off      = enc == ENC_RAW ? nullptr : byte_off;
	c.bw_arr        = enc == ENC_RAW ? nullptr : bw;
	c.base_arr      = base;
	c.lane_base_arr = lane_base;
	c.out           = out;
	return emu_decode_column(&c);
}

// Decode a reference page (host bytes) with the product's host page code + the emulated device logic; with
// cmp != OUT_VALUES, the filter form: out receives one 128-byte bitmap of `value op constant` per vector.
extern "C" int emu_filter_page(const uint8_t* page, uint64_t page_size, const uint8_t* dict, uint64_t dict_size,
                               int value_width, int order, int cmp, uint32_t op, uint64_t value, uint8_t* out);
extern "C" int emu_decode_page(const uint8_t* page, uint64_t page_size, const uint8_t* dict, uint64_t dict_size,
                               int value_width, int order, uint8_t* out) {
	return emu_filter_page(page, page_size, dict, dict_size, value_width, order, OUT_VALUES, 0, 0, out);
}

extern "C" int emu_filter_page(const uint8_t* page, uint64_t page_size, const uint8_t* dict, uint64_t dict_size,
                               int value_width, int order, int cmp, uint32_t op, uint64_t value, uint8_t* out) {
	PageInfo pi;
	int      rc = parse_page_header(page, page_size, &pi);
	if (rc == FLS_OK) { rc = finish_page_info(&pi, page_size); }
	if (rc != FLS_OK) { return -1000 + rc; }
	const uint8_t* dvals   = nullptr;
	uint32_t       entries = 0;
	if (pi.layout->post == POST_DICT || pi.layout->post == POST_RLE_DICT) {
		uint64_t voff = 0;
		rc            = int_dictionary_values(dict, dict_size, value_width, &voff, &entries);
		if (rc != FLS_OK) { return -2000 + rc; }
		dvals = dict + voff;
	}
	ColDesc c;
	rc = build_page_column(pi, page, value_width, dvals, entries, order, out, &c);
	if (rc != FLS_OK) { return -3000 + rc; }
	if (cmp == OUT_VALUES) { return emu_decode_column(&c); }
	c.out_mode = static_cast<uint8_t>(cmp);
	Pred pr {};
	pr.op    = op;
	pr.value = value;
	int st   = 0;
	for (uint32_t v = 0; v < c.n_vec; ++v) { st |= emu_vector(c, v, &pr); }
	return st;
}

// One string through the device FSST / FSST12 row decoders (fls_strings.cuh): its decoded length, and the bytes
// written to out (the length the length pass counts must be what the materialising pass writes).
extern "C" uint64_t emu_fsst_row(int twelve, const uint64_t* sym, const uint8_t* len, const uint8_t* in, uint32_t n,
                                 uint8_t* out) {
	if (twelve) {
		fsst12_decode_to(sym, len, in, n, out);
		return fsst12_decoded_len(len, in, n);
	}
	fsst_decode_to(sym, len, in, n, out);
	return fsst_decoded_len(len, in, n);
}

// A run of FSST rows written to a word window with the string kernels' protocol: the word the first row
// starts in is zeroed, every row's whole words are stored, then the held heads are OR-ed in.  Returns the
// bytes written (the sum of the rows' decoded lengths).
extern "C" uint64_t emu_fsst_put_rows(const uint64_t* sym, const uint8_t* len, const uint8_t* comp,
                                      const uint64_t* coffs, uint32_t n, uint32_t d0, uint32_t* win) {
	win[d0 >> 2]   = 0;
	uint32_t d     = d0;
	std::vector<std::pair<uint32_t, uint32_t>> heads;
	for (uint32_t r = 0; r < n; ++r) {
		const uint8_t* in = comp + coffs[r];
		const uint32_t cn = static_cast<uint32_t>(coffs[r + 1] - coffs[r]);
		uint32_t       hk = 0, head = 0;
		if (fsst_put_row(win, d, sym, len, in, cn, &hk, &head)) { heads.emplace_back(hk, head); }
		d += fsst_decoded_len(len, in, cn);
	}
	for (const auto& h : heads) { win[h.first] |= h.second; }
	return d - d0;
}

// A run of rows copied from the 4-byte aligned word array `base` (row r: bytes [start[r], start[r] + len[r]))
// to a word window with the string kernels' protocol (put_row): returns the bytes written.
extern "C" uint64_t emu_put_rows(const uint32_t* base, const uint32_t* start, const uint32_t* len, uint32_t n,
                                 uint32_t d0, uint32_t* win) {
	win[d0 >> 2] = 0;
	uint32_t d   = d0;
	std::vector<std::pair<uint32_t, uint32_t>> heads;
	for (uint32_t r = 0; r < n; ++r) {
		uint32_t hk = 0, head = 0;
		if (put_row(win, d, base, start[r], len[r], &hk, &head)) { heads.emplace_back(hk, head); }
		d += len[r];
	}
	for (const auto& h : heads) { win[h.first] |= h.second; }
	return d - d0;
}

// One vector of an FSST (fsst = 1) or BYTE_ARR column through the code-parallel device decoder (stream_vector of
// fls_strings.cuh) on an emulated warp: ends = the 1024 cumulative row end offsets (original order), comp / n
// the vector's compressed bytes (at any alignment).  Both passes run: the lengths pass's total is returned in
// *len_total; offsets (1025 values, output positions from vbase) and bytes are written as the materialising
// pass writes them.  Returns the materialising pass's total, *bad whether the rows were refused.
extern "C" uint64_t emu_stream_vector(int fsst, const uint64_t* sym, const uint8_t* len, const uint32_t* ends,
                                      const uint8_t* comp, uint32_t n, uint64_t vbase, uint32_t* offsets, uint8_t* out,
                                      uint64_t* len_total, int* bad_out) {
	std::vector<uint32_t> rows(kVec + kVec / 32 + 32, 0);
	for (uint32_t r = 0; r < kVec; ++r) { rows[r + r / 32] = ends[r]; }
	// the kernel's shared copy of the table: code 255 (the escape) with an empty entry
	std::vector<uint64_t> tsym(256, 0);
	std::vector<uint8_t>  tlen(256, 0);
	if (fsst) {
		for (int c = 0; c < 255; ++c) {
			tsym[c] = sym[c];
			tlen[c] = len[c];
		}
	}
	sym = tsym.data();
	len = tlen.data();
	std::vector<uint8_t> win_buf(2048 + 64, 0xA5);
	uint8_t*             win = reinterpret_cast<uint8_t*>((reinterpret_cast<uintptr_t>(win_buf.data()) + 15) & ~uintptr_t(15));
	uint64_t             tot[2] = {0, 0};
	bool                 bad[2] = {false, false};
	for (int pass = 0; pass < 2; ++pass) {
		std::barrier<>           bar(32);
		EmuWarp                  w {&bar, {}, {}};
		std::vector<std::thread> th;
		for (int t = 0; t < 32; ++t) {
			th.emplace_back([&, t] {
				g_emu_warp = &w;
				g_emu_lane = t;
				StreamOut o {offsets, out, vbase, win};
				bool      b = false;
				uint32_t  r;
				if (pass == 0) {
					r = fsst ? stream_vector<false, true, 2048>(rows.data(), comp, n, sym, len, t, o, &b)
					         : stream_vector<false, false, 2048>(rows.data(), comp, n, sym, len, t, o, &b);
				} else {
					r = fsst ? stream_vector<true, true, 2048>(rows.data(), comp, n, sym, len, t, o, &b)
					         : stream_vector<true, false, 2048>(rows.data(), comp, n, sym, len, t, o, &b);
				}
				if (t == 0) {
					tot[pass] = r;
					bad[pass] = b;
				}
			});
		}
		for (auto& x : th) { x.join(); }
	}
	offsets[kVec] = static_cast<uint32_t>(vbase + tot[1]);
	*len_total    = tot[0];
	*bad_out      = (bad[0] ? 1 : 0) | (bad[1] ? 2 : 0);
	return tot[1];
}

// fsst_plain_total (fls_strings.cuh) on an emulated warp: the bytes [0, L) at vb (any alignment), len the 256
// symbol lengths (code 255's taken as 0, as the kernels' shared copy has it).  Returns 1 when the function
// reports no escape (then *total is its sum), 0 otherwise.
extern "C" int emu_fsst_plain_total(const uint8_t* len, const uint8_t* vb, uint32_t L, uint32_t* total) {
	std::vector<uint8_t> tlen(256, 0);
	for (int c = 0; c < 255; ++c) { tlen[c] = len[c]; }
	std::barrier<>           bar(32);
	EmuWarp                  w {&bar, {}, {}};
	std::vector<std::thread> th;
	int                      plain = 0;
	uint32_t                 tot   = 0;
	for (int t = 0; t < 32; ++t) {
		th.emplace_back([&, t] {
			g_emu_warp = &w;
			g_emu_lane = t;
			uint32_t   x  = 0;
			const bool ok = fsst_plain_total(vb, L, tlen.data(), t, &x);
			if (t == 0) {
				plain = ok ? 1 : 0;
				tot   = x;
			}
		});
	}
	for (auto& x : th) { x.join(); }
	*total = tot;
	return plain;
}
