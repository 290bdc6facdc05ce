// Test infrastructure only: a stand-in for the un-vendored ALP header (github.com/cwida/ALP, tag "main",
// not present in the reference snapshot). The reference includes "alp.hpp" from src/cor/eng/analyzer.cpp:2
// and only touches ALP on the double-precision path, which is outside the integer/string decode path this
// oracle is built for. Every member is a no-op; the ALP compress/decompress primitives are not compiled.
#ifndef FLS_ORACLE_ALP_SHIM_HPP
#define FLS_ORACLE_ALP_SHIM_HPP

#include <cstddef>
#include <cstdint>

namespace alp {
template <typename T>
struct state {
	uint8_t exp {0};
	uint8_t fac {0};
};

template <typename T>
struct encoder {
	template <typename... A>
	static void init(A&&...) {}
	template <typename... A>
	static void encode(A&&...) {}
	template <typename... A>
	static void analyze_ffor(A&&...) {}
};
} // namespace alp

#endif
