// Test infrastructure only. Replaces src/cor/prm/alp/alp_{compress,decompress}.cpp of the reference, which
// need the external ALP library. The resolver (src/cor/eng/resolver.cpp:214,361) links against these two
// function templates; on the integer/string path they are never called, so they resolve to nullptr.
#include <cstdint>
#include "fls/cor/prm/alp_prm.hpp"

namespace fastlanes {
template <typename T>
cmpr_fun_t alp_prm::ResolveCompressFunc() {
	return nullptr;
}
template <typename T>
de_cmpr_fun_t alp_prm::ResolveDecompressFunc() {
	return nullptr;
}
template cmpr_fun_t    alp_prm::ResolveCompressFunc<double>();
template de_cmpr_fun_t alp_prm::ResolveDecompressFunc<double>();
} // namespace fastlanes
