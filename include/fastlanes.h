/* fastlanes.h — the reference's C API (cwida/FastLanes include/fastlanes.h:14-111), served by the B200 engine.
 *
 * Same names, argument meaning and enum values as the reference, so a program written against the reference
 * links against libfls_b200.so unchanged.  encode_from_memory encodes on the GPU and frames the result as a
 * FastLanes page (bit-identical to the reference's page for the same input); decode_to_memory decodes on the
 * GPU.  Both take HOST pointers and copy through device memory.  Besides the reference's INT64 expressions
 * 0 (UNCOMPRESSED), 1 (FFOR) and 11 (DELTA), the engine encodes expression 6 (RLE DELTA_NO_PATCH, the pool
 * id of src/cor/exp_pool.cpp:31) and accepts UINT32 / INT32 / UINT64 columns with the same framing
 * (T = the 32/64-bit type).
 */
#ifndef FASTLANES_H
#define FASTLANES_H

#include <stdbool.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* datatype — values of include/fastlanes.h:14-34 */
enum data_t : uint8_t {
	INVALID    = 0,
	DOUBLE     = 1,
	INT8       = 2,
	INT16      = 3,
	INT32      = 4,
	INT64      = 5,
	UINT8      = 6,
	UINT16     = 7,
	UINT32     = 8,
	UINT64     = 9,
	STR        = 10,
	BOOLEAN    = 11,
	DATE       = 12,
	FLOAT      = 13,
	BYTE_ARRAY = 14,
	LIST       = 15,
	STRUCT     = 16,
	MAP        = 17,
	FALLBACK   = 18,
};

/* int64 expression ids — include/fastlanes.h:37-41 */
enum i64_expr_encoding_t : uint8_t {
	I64_UNCOMPRESSED   = 0,
	I64_FFOR_NO_PATCH  = 1,
	I64_DELTA_NO_PATCH = 11,
};

/* double expression ids — include/fastlanes.h:44-47 (ALP is outside the decode path of this engine) */
enum dbl_expr_encoding_t : uint8_t {
	DBL_UNCOMPRESSED = 0,
	DBL_ALP          = 1,
};

typedef struct Connection connection_cpi;

/* include/fastlanes.h:53-54 */
connection_cpi* fls_cpi_connection_open();
void            fls_cpi_connection_close(connection_cpi* fls_connection);

/* include/fastlanes.h:72-79: encode in_n_input values (whole 1024-value vectors; a tail of n % 1024 values is
 * dropped, as the reference's encoder does).  Returns false when the encoded page does not fit in_capacity or
 * the type / expression is not supported.  out_metadadata_size receives the page's header + offsets + entry
 * points size. */
bool encode_from_memory(void*       in_data,
                        uint64_t    in_n_input,
                        uint64_t    in_capacity,
                        uint8_t*    out_encoded_data,
                        uint64_t*   out_encoded_size,
                        uint64_t*   out_metadadata_size,
                        enum data_t in_datatype,
                        uint8_t     in_expression_type);

/* include/fastlanes.h:84-86: decode a page into vec_c * 1024 values (original order). */
void decode_to_memory(uint8_t* in_encoded_data, void* out_data, enum data_t in_datatype);

/* include/fastlanes.h:88-108 (declared by the reference, defined nowhere there).  Random access to one vector
 * of an INT64 page whose buffers are all per vector (expressions 0, 1, 11, RLE 6, patched FFOR / DELTA without
 * rec buffers); other pages report no buffers / leave the output untouched.
 * init_random_access: with the page's metadata (header, buffer offsets, entry points) loaded at
 *   in_encoded_data, the buffers vector in_vector_id needs: *output_n_buffer pairs [offset, size] (bytes from
 *   the page start) in output_buffer (room for 2 * 6 values).  The last vector's packed buffer is reported with
 *   the largest size a vector can take (8192 bytes); a caller clips it to the page.
 * random_access: decodes vector in_vector_id into out_deencoded_vector (1024 int64 values, original order)
 *   from the loaded buffers output_buffers[i] (the ranges init_random_access gave). */
void init_random_access(uint8_t* in_encoded_data, uint64_t in_vector_id, uint64_t* output_n_buffer,
                        uint64_t* output_buffer);
void random_access(uint8_t* in_encoded_data, uint64_t in_vector_id, uint64_t* output_n_buffer,
                   uint64_t* output_pair_offset_and_size, uint8_t** output_buffers, uint8_t* out_deencoded_vector);

/* Status-returning forms of the two random-access calls (0 = ok, fls_status_code of fls_b200.h otherwise). */
int fls_random_access_ranges(const uint8_t* in_encoded_data, uint64_t in_vector_id, uint64_t* n_buffer,
                             uint64_t* pairs);
int fls_random_access_decode(const uint8_t* in_encoded_data, uint64_t in_vector_id, uint64_t n_buffer,
                             const uint64_t* pairs, const uint8_t* const* buffers, int64_t* out);

/* Status-returning forms of encode_from_memory / decode_to_memory (0 = ok, fls_status_code of fls_b200.h otherwise).
 * fls_decode_to_memory_checked also bounds the input by in_encoded_size and reports the vector count. */
int fls_encode_from_memory_status(void* in_data, uint64_t in_n_input, uint64_t in_capacity, uint8_t* out_encoded_data,
                                  uint64_t* out_encoded_size, uint64_t* out_metadadata_size, enum data_t in_datatype,
                                  uint8_t in_expression_type);
int fls_decode_to_memory_checked(const uint8_t* in_encoded_data, uint64_t in_encoded_size, void* out_data,
                                 uint64_t out_capacity_bytes, enum data_t in_datatype, uint64_t* out_n_values);

#ifdef __cplusplus
}
#endif

#endif /* FASTLANES_H */
