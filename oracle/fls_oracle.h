/* TEST INFRASTRUCTURE — the CPU oracle for the FastLanes decode path.
 *
 * A plain-C restatement of the reference's scalar primitives and column framing, used only by tests/,
 * __graft_entry__.smoke() and bench.py's cpu_baseline leg as the checker.  The product library never links
 * it.  Parity is pinned against the reference's own golden vectors (tests/golden/, made from
 * primitives/fls_generated/fallback/scalar_aav_uf1/ *_helper.hpp files) and against the reference compiled from
 * its sources (oracle/_ref/libfls_ref.so).
 *
 * Every routine works on one 1024-value vector in the FastLanes unified transposed layout:
 *   transposed[k] = original[(k % 16) * 64 + O[(k / 16) % 8] * 8 + k / 128],  O = {0,4,2,6,1,5,3,7}
 * A W-bit type has L = 1024 / W lanes; lane i's packed word w is in[i + L*w]; lane i's value j sits at
 * transposed position i + L*j.  Bits are LSB-first within a word and a value may straddle two words.
 */
#ifndef FLS_ORACLE_H
#define FLS_ORACLE_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

uint32_t fls_o_original_index(uint32_t k);

#define FLS_O_DECL(T, S)                                                                                       \
	void    fls_o_transpose_i_##S(const T* in, T* out);                                                      \
	void    fls_o_untranspose_i_##S(const T* in, T* out);                                                    \
	void    fls_o_pack_##S(const T* in, T* out, uint8_t bw);                                                 \
	void    fls_o_unpack_##S(const T* in, T* out, uint8_t bw);                                               \
	void    fls_o_ffor_##S(const T* in, T* out, uint8_t bw, const T* base);                                  \
	void    fls_o_unffor_##S(const T* in, T* out, uint8_t bw, const T* base);                                \
	void    fls_o_rsum_##S(const T* in, T* out, const T* base);                                              \
	void    fls_o_unrsum_##S(const T* in, T* out);                                                           \
	uint8_t fls_o_analyze_##S(const T* in, T* base_out);                                                     \
	void    fls_o_unffor_batch_##S(const T* packed, const uint64_t* word_off, const uint8_t* bw, const T* base, \
	                               uint64_t n_vec, int original_order, T* out);

FLS_O_DECL(uint8_t, u8)
FLS_O_DECL(uint16_t, u16)
FLS_O_DECL(uint32_t, u32)
FLS_O_DECL(uint64_t, u64)

/* FSST decode of one string with an imported symbol table, restating fsst_decompress
 * (include/fls/cor/prm/fsst/fsst.h:152-259).  sym[c] holds symbol c little-endian, len[c] its length;
 * code 255 is the escape.  Returns the decoded length (which may exceed cap; only cap bytes are written). */
uint64_t fls_o_fsst_decode(const uint64_t* sym, const uint8_t* len, const uint8_t* in, uint64_t in_len,
                           uint8_t* out, uint64_t cap);

/* Import an FSST symbol table written by fsst_export (src/cor/prm/fsst/libfsst.cpp:617-657).
 * Returns the number of header bytes consumed, 0 on a malformed header. */
uint32_t fls_o_fsst_import(const uint8_t* buf, uint64_t* sym, uint8_t* len);

/* FSST12 decode of one string, restating fsst12_decompress (include/fls/cor/prm/fsst12/fsst12.h:130-177):
 * every 3 input bytes hold two 12-bit codes (little-endian), a trailing 2 bytes one code; no escapes.
 * sym/len hold 4096 codes.  Returns the decoded length (only cap bytes are written). */
uint64_t fls_o_fsst12_decode(const uint64_t* sym, const uint8_t* len, const uint8_t* in, uint64_t in_len,
                             uint8_t* out, uint64_t cap);

/* Import an FSST12 symbol table written by fsst12_export (src/cor/prm/fsst12/libfsst12.cpp:363-389).
 * Returns the number of header bytes consumed, 0 on a malformed header. */
uint32_t fls_o_fsst12_import(const uint8_t* buf, uint64_t avail, uint64_t* sym, uint8_t* len);

#ifdef __cplusplus
}
#endif
#endif
