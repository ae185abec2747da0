// tests/fftm.cpp and tests/fft.cpp of the reference call error_db(), which no
// header of the reference declares (the reference's own build fails on it).
// This shim maps it to the reference's test metric test::diff
// (support/test/diff.hpp:41-96) so those tests compile unmodified.
#ifndef FCB200_ERROR_DB_SHIM_HPP
#define FCB200_ERROR_DB_SHIM_HPP
#include <test.hpp>
namespace vsip
{
template <typename V1, typename V2>
double error_db(V1 const &v1, V2 const &v2) { return ::test::diff(v1, v2); }
}
#endif
