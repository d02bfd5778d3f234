/*
 * The reference's IPM vector header only needs two scalar helpers from its
 * autodiff dependency.  This oracle-only stand-in defines them from their
 * plain meaning (the smaller / larger of two values).
 */
#ifndef ORACLE_A2DCORE_STUB_H
#define ORACLE_A2DCORE_STUB_H
namespace A2D {
template <typename T>
inline T min2(T a, T b) { return a < b ? a : b; }
template <typename T>
inline T max2(T a, T b) { return a > b ? a : b; }
}  // namespace A2D
#endif
