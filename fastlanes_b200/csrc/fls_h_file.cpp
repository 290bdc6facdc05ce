// Files: the reference's file pair data.fls + footer.json (Connection::to_fls, src/connection.cpp:102-128;
// Reader, src/reader/reader.cpp:19-61; footer keys of src/json/fls_json.cpp:30-62) read into device memory.
//
// The reference stores a column's values only for its ZERO_COPY columns (n_vec * 1024 raw values at col_ofs,
// src/expression/store_operator.cpp:24-35); its CONSTANT and EQUAL columns keep neither the constant nor the
// equal column's index in the footer, so they cannot be read back (its own Reader does not try).  This
// library adds page columns in the same container: a "pages" list in the column's metadata, each entry one
// row-group chunk {"ofs", "size", "dict_ofs", "dict_size", "n_vec"} of reference page bytes, decoded on the
// GPU by one page decode over every chunk of every requested column.
#include "fls_b200.h"
#include "fastlanes.h"
#include "fls_runtime.h"

#include <cuda_runtime.h>

#include <algorithm>
#include <cstdio>
#include <cstring>
#include <fcntl.h>
#include <memory>
#include <string>
#include <unistd.h>
#include <vector>

namespace {

// ---- a small JSON reader (objects, arrays, strings, integers, true / false / null) ---------------------
struct JVal {
	enum Kind { NUL, BOOL, NUM, STR, ARR, OBJ } kind = NUL;
	bool                                      b    = false;
	int64_t                                   i    = 0;
	uint64_t                                  u    = 0;
	bool                                      neg  = false;
	std::string                               s;
	std::vector<JVal>                         arr;
	std::vector<std::pair<std::string, JVal>> obj;

	const JVal* get(const char* key) const {
		for (const auto& kv : obj) {
			if (kv.first == key) { return &kv.second; }
		}
		return nullptr;
	}
};

struct JParser {
	const char* p;
	const char* e;
	int         depth = 0;

	void ws() {
		while (p < e && (*p == ' ' || *p == '\n' || *p == '\r' || *p == '\t')) { ++p; }
	}
	bool lit(const char* w) {
		const size_t n = std::strlen(w);
		if (static_cast<size_t>(e - p) < n || std::memcmp(p, w, n) != 0) { return false; }
		p += n;
		return true;
	}
	bool str(std::string* out) {
		if (p >= e || *p != '"') { return false; }
		++p;
		while (p < e && *p != '"') {
			if (*p == '\\') {
				if (++p >= e) { return false; }
				switch (*p) {
				case 'n': out->push_back('\n'); break;
				case 't': out->push_back('\t'); break;
				case 'r': out->push_back('\r'); break;
				case 'b': out->push_back('\b'); break;
				case 'f': out->push_back('\f'); break;
				case 'u': // \uXXXX: kept as '?' (the footer's keys and names are ASCII)
					if (e - p < 5) { return false; }
					p += 4;
					out->push_back('?');
					break;
				default: out->push_back(*p);
				}
				++p;
			} else {
				out->push_back(*p++);
			}
		}
		if (p >= e) { return false; }
		++p;
		return true;
	}
	bool val(JVal* v) {
		if (++depth > 64) { return false; }
		ws();
		if (p >= e) { return false; }
		bool ok = true;
		if (*p == '{') {
			v->kind = JVal::OBJ;
			++p;
			ws();
			if (p < e && *p == '}') {
				++p;
			} else {
				while (ok) {
					ws();
					std::string k;
					JVal        x;
					ok = str(&k);
					ws();
					ok = ok && p < e && *p++ == ':' && val(&x);
					if (ok) { v->obj.emplace_back(std::move(k), std::move(x)); }
					ws();
					if (!ok || p >= e) { return false; }
					if (*p == ',') {
						++p;
					} else if (*p == '}') {
						++p;
						break;
					} else {
						return false;
					}
				}
			}
		} else if (*p == '[') {
			v->kind = JVal::ARR;
			++p;
			ws();
			if (p < e && *p == ']') {
				++p;
			} else {
				while (ok) {
					JVal x;
					ok = val(&x);
					if (ok) { v->arr.push_back(std::move(x)); }
					ws();
					if (!ok || p >= e) { return false; }
					if (*p == ',') {
						++p;
					} else if (*p == ']') {
						++p;
						break;
					} else {
						return false;
					}
				}
			}
		} else if (*p == '"') {
			v->kind = JVal::STR;
			ok      = str(&v->s);
		} else if (lit("true")) {
			v->kind = JVal::BOOL, v->b = true;
		} else if (lit("false")) {
			v->kind = JVal::BOOL;
		} else if (lit("null")) {
			v->kind = JVal::NUL;
		} else {
			v->kind = JVal::NUM;
			if (*p == '-') { v->neg = true, ++p; }
			if (p >= e || *p < '0' || *p > '9') { return false; }
			while (p < e && *p >= '0' && *p <= '9') {
				const uint64_t d = static_cast<uint64_t>(*p - '0');
				if (v->u > (UINT64_MAX - d) / 10) { return false; }
				v->u = v->u * 10 + d;
				++p;
			}
			if (p < e && (*p == '.' || *p == 'e' || *p == 'E')) { return false; } // the footer has integers only
			v->i = v->neg ? -static_cast<int64_t>(v->u) : static_cast<int64_t>(v->u);
		}
		--depth;
		return ok;
	}
};

bool read_file(const std::string& path, std::string* out) {
	FILE* f = std::fopen(path.c_str(), "rb");
	if (!f) { return false; }
	char   b[65536];
	size_t n = 0;
	while ((n = std::fread(b, 1, sizeof(b), f)) > 0) { out->append(b, n); }
	const bool ok = std::ferror(f) == 0;
	std::fclose(f);
	return ok;
}

int value_bytes(uint8_t t) {
	switch (t) {
	case INT64:
	case UINT64:
	case DOUBLE: return 8;
	case INT32:
	case UINT32: return 4;
	case INT16:
	case UINT16: return 2;
	case INT8:
	case UINT8: return 1;
	default: return 0;
	}
}

struct PageRef {
	uint64_t ofs, size, dict_ofs, dict_size, n_vec;
};

} // namespace

struct fls_file {
	std::string          data_path;
	uint64_t             n_vec    = 0;
	uint64_t             rg_size  = 0;
	uint64_t             fsize    = 0;
	struct Col {
		uint8_t              type = 0, kind = FLS_FILE_NO_DATA;
		uint64_t             ofs  = 0;
		uint64_t             n_vec = 0;
		std::vector<PageRef> pages;
	};
	std::vector<Col> cols;
};

extern "C" {

int fls_file_open(const char* dir, fls_file** out) {
	if (!dir || !out) { return FLS_ERR_ARG; }
	*out = nullptr;
	const std::string d(dir);
	std::string       js;
	if (!read_file(d + "/footer.json", &js)) { return FLS_ERR_ARG; }
	JVal    root;
	JParser jp {js.data(), js.data() + js.size()};
	if (!jp.val(&root) || root.kind != JVal::OBJ) { return FLS_ERR_FORMAT; }
	const JVal* nv   = root.get("1: N VEC");
	const JVal* rs   = root.get("2: Rowgroup size");
	const JVal* mtds = root.get("3: Column Metadatas");
	if (!nv || nv->kind != JVal::NUM || nv->neg || !mtds || mtds->kind != JVal::ARR) { return FLS_ERR_FORMAT; }
	std::unique_ptr<fls_file> f(new fls_file());
	f->data_path = d + "/data.fls";
	f->n_vec     = nv->u;
	f->rg_size   = rs && rs->kind == JVal::NUM ? rs->u : 0;
	{
		FILE* fp = std::fopen(f->data_path.c_str(), "rb");
		if (!fp) { return FLS_ERR_ARG; }
		std::fseek(fp, 0, SEEK_END);
		const long sz = std::ftell(fp);
		std::fclose(fp);
		if (sz < 0) { return FLS_ERR_ARG; }
		f->fsize = static_cast<uint64_t>(sz);
	}
	for (const JVal& m : mtds->arr) {
		if (m.kind != JVal::OBJ) { return FLS_ERR_FORMAT; }
		fls_file::Col c;
		const JVal*   lt  = m.get("logical_type");
		const JVal*   ofs = m.get("col_ofs");
		const JVal*   rpn = m.get("Encoding RPN");
		if (!lt || lt->kind != JVal::NUM || !ofs || ofs->kind != JVal::NUM) { return FLS_ERR_FORMAT; }
		c.type  = static_cast<uint8_t>(lt->u);
		c.ofs   = ofs->u;
		c.n_vec = f->n_vec;
		const JVal* ops = rpn ? rpn->get("operators") : nullptr;
		std::string op0;
		if (ops && ops->kind == JVal::ARR && !ops->arr.empty() && ops->arr[0].kind == JVal::STR) { op0 = ops->arr[0].s; }
		const int w = value_bytes(c.type);
		if (op0 == "ZERO_COPY" && w > 0) {
			c.kind = FLS_FILE_ZERO_COPY;
			if (c.ofs > f->fsize || f->n_vec * 1024ull * w > f->fsize - c.ofs) { return FLS_ERR_FORMAT; }
		} else if (op0 == "FLS_PAGES" && w > 0) {
			c.kind = FLS_FILE_PAGES;
			const JVal* pg = m.get("pages");
			if (!pg || pg->kind != JVal::ARR) { return FLS_ERR_FORMAT; }
			c.n_vec = 0;
			for (const JVal& x : pg->arr) {
				PageRef     r {};
				const char* keys[5] = {"ofs", "size", "dict_ofs", "dict_size", "n_vec"};
				uint64_t*   dst[5]  = {&r.ofs, &r.size, &r.dict_ofs, &r.dict_size, &r.n_vec};
				for (int k = 0; k < 5; ++k) {
					const JVal* y = x.get(keys[k]);
					if (!y || y->kind != JVal::NUM || y->neg) { return FLS_ERR_FORMAT; }
					*dst[k] = y->u;
				}
				if (r.ofs > f->fsize || r.size > f->fsize - r.ofs || r.dict_ofs > f->fsize ||
				    r.dict_size > f->fsize - r.dict_ofs || r.n_vec == 0 || r.n_vec > 65535) {
					return FLS_ERR_FORMAT;
				}
				c.pages.push_back(r);
				c.n_vec += r.n_vec;
			}
		} else {
			c.kind = FLS_FILE_NO_DATA; // CONSTANT, EQUAL, ...: the reference keeps no values for them
		}
		f->cols.push_back(std::move(c));
	}
	*out = f.release();
	return FLS_OK;
}

int fls_file_shape(const fls_file* f, uint32_t* n_cols, uint64_t* n_vec) {
	if (!f || !n_cols || !n_vec) { return FLS_ERR_ARG; }
	*n_cols = static_cast<uint32_t>(f->cols.size());
	*n_vec  = f->n_vec;
	return FLS_OK;
}

int fls_file_column(const fls_file* f, uint32_t col, uint8_t* data_type, uint8_t* kind, uint64_t* n_values) {
	if (!f || col >= f->cols.size() || !data_type || !kind || !n_values) { return FLS_ERR_ARG; }
	const auto& c = f->cols[col];
	*data_type    = c.type;
	*kind         = c.kind;
	*n_values     = c.kind == FLS_FILE_NO_DATA ? 0 : c.n_vec * 1024;
	return FLS_OK;
}

int fls_file_read(fls_file* f, const uint32_t* cols, uint32_t n, void* const* d_outs, fls_stream_t stream) {
	if (!f || (n && (!cols || !d_outs))) { return FLS_ERR_ARG; }
	cudaStream_t s = static_cast<cudaStream_t>(stream);
	uint64_t     page_bytes = 0, n_pages = 0, max_piece = 1 << 20;
	for (uint32_t i = 0; i < n; ++i) {
		if (cols[i] >= f->cols.size() || !d_outs[i]) { return FLS_ERR_ARG; }
		const auto& c = f->cols[cols[i]];
		if (c.kind == FLS_FILE_NO_DATA) { return FLS_ERR_UNSUPPORTED; }
		if (c.kind == FLS_FILE_PAGES && c.type == DOUBLE) { return FLS_ERR_UNSUPPORTED; }
		for (const auto& r : c.pages) {
			page_bytes += ((r.size + 15) & ~15ull) + 16 + ((r.dict_size + 15) & ~15ull) + 16;
			max_piece = std::max<uint64_t>(max_piece, std::max(r.size, r.dict_size));
			++n_pages;
		}
	}
	if (n_pages > 65535) { return FLS_ERR_ARG; }
	const int fd = ::open(f->data_path.c_str(), O_RDONLY);
	if (fd < 0) { return FLS_ERR_ARG; }
	// two pinned bounce buffers: the file read into one overlaps the copy out of the other
	const uint64_t kChunk = std::max<uint64_t>(32ull << 20, max_piece);
	uint8_t*       bounce[2] {};
	cudaEvent_t    done[2] {};
	uint8_t*       staging = nullptr;
	int            rc      = FLS_OK;
	auto           fail    = [&](int code) {
		if (rc == FLS_OK) { rc = code; }
	};
	for (int k = 0; k < 2; ++k) {
		if (cudaHostAlloc(reinterpret_cast<void**>(&bounce[k]), kChunk, cudaHostAllocDefault) != cudaSuccess ||
		    cudaEventCreateWithFlags(&done[k], cudaEventDisableTiming) != cudaSuccess) {
			fail(FLS_ERR_CUDA);
		}
	}
	int turn = 0;
	// file bytes [ofs, ofs + size) to device dst, through the bounce buffers
	auto stream_in = [&](uint64_t ofs, uint64_t size, uint8_t* dst) {
		uint64_t done_b = 0;
		while (rc == FLS_OK && done_b < size) {
			const uint64_t take = std::min(kChunk, size - done_b);
			if (cudaEventSynchronize(done[turn]) != cudaSuccess) { return fail(FLS_ERR_CUDA); }
			uint64_t got = 0;
			while (got < take) {
				const ssize_t r = ::pread(fd, bounce[turn] + got, take - got, static_cast<off_t>(ofs + done_b + got));
				if (r <= 0) { return fail(FLS_ERR_FORMAT); }
				got += static_cast<uint64_t>(r);
			}
			if (cudaMemcpyAsync(dst + done_b, bounce[turn], take, cudaMemcpyHostToDevice, s) != cudaSuccess ||
			    cudaEventRecord(done[turn], s) != cudaSuccess) {
				return fail(FLS_ERR_CUDA);
			}
			turn ^= 1;
			done_b += take;
		}
	};
	if (rc == FLS_OK && page_bytes && cudaMalloc(reinterpret_cast<void**>(&staging), page_bytes + 64) != cudaSuccess) {
		fail(FLS_ERR_CUDA);
	}
	std::vector<fls_page_column> pcs;
	uint64_t                     pos = 0;
	for (uint32_t i = 0; i < n && rc == FLS_OK; ++i) {
		const auto&    c = f->cols[cols[i]];
		const uint64_t w = static_cast<uint64_t>(value_bytes(c.type));
		uint8_t*       o = static_cast<uint8_t*>(d_outs[i]);
		if (c.kind == FLS_FILE_ZERO_COPY) {
			stream_in(c.ofs, c.n_vec * 1024 * w, o);
			continue;
		}
		uint64_t first_vec = 0;
		for (const auto& r : c.pages) {
			// the page lands 16-byte aligned plus the shift that puts its packed buffer on a 16-byte boundary
			uint8_t  pre[64] {};
			uint8_t* base = staging + pos;
			uint32_t shift = 0;
			{
				uint64_t       got  = 0;
				const uint64_t want = std::min<uint64_t>(sizeof(pre), r.size);
				while (got < want) {
					const ssize_t x = ::pread(fd, pre + got, want - got, static_cast<off_t>(r.ofs + got));
					if (x <= 0) { break; }
					got += static_cast<uint64_t>(x);
				}
				if (got < want || fls_page_placement(pre, want, &shift) != FLS_OK) { shift = 0; }
			}
			stream_in(r.ofs, r.size, base + shift);
			pos += ((r.size + 15) & ~15ull) + 16;
			uint8_t* dict = nullptr;
			if (r.dict_size) {
				dict = staging + pos;
				stream_in(r.dict_ofs, r.dict_size, dict);
				pos += ((r.dict_size + 15) & ~15ull) + 16;
			}
			fls_page_column pc {};
			pc.d_page    = base + shift;
			pc.page_size = r.size;
			pc.d_dict    = dict;
			pc.dict_size = r.dict_size;
			pc.data_type = c.type;
			pc.order     = FLS_ORIGINAL;
			pc.d_out     = o + first_vec * 1024 * w;
			pcs.push_back(pc);
			first_vec += r.n_vec;
		}
	}
	if (rc == FLS_OK && !pcs.empty()) {
		// every chunk of every requested page column in one decode (one launch per kernel class)
		const int d = fls_gpu_decode_pages(pcs.data(), static_cast<uint32_t>(pcs.size()), stream);
		if (d != FLS_OK) { fail(d); }
	}
	if (cudaStreamSynchronize(s) != cudaSuccess) { fail(FLS_ERR_CUDA); }
	for (int k = 0; k < 2; ++k) {
		if (done[k]) { cudaEventDestroy(done[k]); }
		if (bounce[k]) { cudaFreeHost(bounce[k]); }
	}
	if (staging) { cudaFree(staging); }
	::close(fd);
	return rc;
}

int fls_file_close(fls_file* f) {
	delete f;
	return FLS_OK;
}

} // extern "C"
