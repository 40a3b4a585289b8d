// Thin C wrapper around the reference's own lo_float.h, compiled from the
// reference source tree by oracle/Makefile (target `ref`) into oracle/_ref/.
// TEST INFRASTRUCTURE ONLY: it generates/validates golden conversion vectors.
// Calls lo_float::float8_e4m3fn / float8_e5m2 ::ConvertFrom<kSaturate, kTruncate=false>
// (src/lo_float.h:2122-2131 -> ConvertImpl::run, src/lo_float.h:1960-2120), and the
// float6_e2m3 / float6_e3m2 / float4_e2m1 conversions (src/lo_float.h:603-645), whose
// decoded values are returned.
#include "lo_float.h"
#include <cstdint>

extern "C" {
void ref_lofloat_e4m3(const float* x, uint8_t* out, long long n, int saturate) {
  for (long long i = 0; i < n; ++i)
    out[i] = saturate ? lo_float::float8_e4m3fn::ConvertFrom<true, false>(x[i]).rep()
                      : lo_float::float8_e4m3fn::ConvertFrom<false, false>(x[i]).rep();
}
void ref_lofloat_e5m2(const float* x, uint8_t* out, long long n, int saturate) {
  for (long long i = 0; i < n; ++i)
    out[i] = saturate ? lo_float::float8_e5m2::ConvertFrom<true, false>(x[i]).rep()
                      : lo_float::float8_e5m2::ConvertFrom<false, false>(x[i]).rep();
}
// saturating RNE conversions to the 6- and 4-bit types, as float values
void ref_lofloat_f6e2m3(const float* x, float* out, long long n) {
  for (long long i = 0; i < n; ++i) out[i] = (float)lo_float::float6_e2m3::ConvertFrom<true, false>(x[i]);
}
void ref_lofloat_f6e3m2(const float* x, float* out, long long n) {
  for (long long i = 0; i < n; ++i) out[i] = (float)lo_float::float6_e3m2::ConvertFrom<true, false>(x[i]);
}
void ref_lofloat_f4e2m1(const float* x, float* out, long long n) {
  for (long long i = 0; i < n; ++i) out[i] = (float)lo_float::float4_e2m1::ConvertFrom<true, false>(x[i]);
}
}
