// Page metadata and the expression table shared by the host modules.
#pragma once

#include "fls_plan.h"
#include <cuda_runtime.h>
#include <cstdint>

namespace flsgpu {

struct ExprLayout {
	uint8_t exp_t, var, arr_c;
	uint8_t ws; // stream width in bits; 0 = the column's value width
	uint8_t enc, post;
	uint8_t ib_bw, ib_base, ib_packed, ib_lane, ib_vals;
	uint8_t ib_rec;          // the rec-compressed buffer of the ..._REC variants (kNoBuf: none)
	uint8_t ib_exc, ib_side; // patched variants: exception values, positions / bitmap / chain head
	uint8_t dict_codes;      // 1: the patched stream is u32 dictionary codes, gathered from the dictionary after
	uint8_t ib_rec2 = kNoBuf; // a second rec-compressed buffer (RLE REC2: the u16 rsum bases)
};

struct PageInfo {
	uint8_t           exp_t = 0, var = 0;
	uint16_t          vec_c = 0;
	uint32_t          arr_c = 0;
	uint32_t          off[6] {};
	uint64_t          size[6] {};
	uint64_t          ep_off  = 0;
	uint64_t          meta_sz = 0;
	const ExprLayout* layout  = nullptr;
};

const ExprLayout* expr_layout(uint8_t exp_t, uint8_t var);
int               value_width_of(uint8_t data_type);
int               parse_page_header(const uint8_t* hdr, uint64_t avail, PageInfo* out);
int               finish_page_info(PageInfo* pi, uint64_t page_size);
// d_vals_decoded / vals_decoded_size: for the _REC layouts, the decoded rec buffer that replaces buffer ib_rec;
// d_rec2 / rec2_size: the decoded second rec buffer (ib_rec2) of the REC2 layout.
int build_page_column(const PageInfo& pi, const uint8_t* d_page, int value_width, const uint8_t* d_dict_vals,
                      uint32_t dict_entries, int order, uint8_t* d_out, ColDesc* c,
                      const uint8_t* d_vals_decoded = nullptr, uint64_t vals_decoded_size = 0,
                      const uint8_t* d_rec2 = nullptr, uint64_t rec2_size = 0);
// The u32 code stream of a DICT / DICT_FRQ page whose codes are patched FFOR / DELTA streams (page bytes in
// device memory) decoded into d_codes (vec_c * 1024 u32, transposed order, as an UNCOMPRESSED page stores
// them), exceptions rec-decoded first where the variant compresses them.  Synchronises `stream`.
int decode_patched_codes(const uint8_t* d_page, uint64_t page_size, uint32_t* d_codes, cudaStream_t stream);
// RLE DELTA_NO_PATCH page (fls_h_encode.cpp) of n values of width 32 or 64 from host memory.
int encode_rle_page(const void* in, uint64_t n, uint64_t cap, uint8_t* out, uint64_t* out_size, uint64_t* mtd_size,
                    int width);
int int_dictionary_values(const uint8_t* dict, uint64_t dict_size, int value_width, uint64_t* vals_off,
                          uint32_t* entries);

} // namespace flsgpu
