// Thrust 2.x removed pinned_allocator; the codec only needs an allocator type.
#pragma once
#include <memory>
namespace thrust { namespace system { namespace cuda { namespace experimental {
template <class T> using pinned_allocator = std::allocator<T>;
}}}}
