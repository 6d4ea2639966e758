// Stand-in for the moderngpu header the reference includes (moderngpu is not vendored).
// Only the names cm.h mentions are declared; nothing here is called by the codec.
#pragma once
namespace mgpu {
struct standard_context_t {};
template <class T> struct plus_t {};
template <class T> struct minimum_t {};
template <class T> struct maximum_t {};
template <class T> struct less_t {};
}  // namespace mgpu
