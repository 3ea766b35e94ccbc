// Project-written stand-in for waLBerla's core/DataTypes.h: the integer/real typedefs and
// no-op assertion macros the reference's generated kernels and index headers refer to.
// Test infrastructure only (oracle/_ref build).
#pragma once
#include <cstddef>
#include <cstdint>
namespace walberla {
typedef std::size_t uint_t;
typedef double real_t;
typedef std::uint16_t uint16_t;
template <typename T> inline real_t real_c(T t) { return static_cast<real_t>(t); }
template <typename T> inline uint_t uint_c(T t) { return static_cast<uint_t>(t); }
template <typename T> inline int int_c(T t) { return static_cast<int>(t); }
}  // namespace walberla
#define WALBERLA_UNUSED(x) (void)(x)
#define WALBERLA_ASSERT(...) ((void)0)
#define WALBERLA_ASSERT_EQUAL(...) ((void)0)
#define WALBERLA_ASSERT_UNEQUAL(...) ((void)0)
#define WALBERLA_ASSERT_LESS(...) ((void)0)
#define WALBERLA_ASSERT_LESS_EQUAL(...) ((void)0)
#define WALBERLA_ASSERT_GREATER(...) ((void)0)
#define WALBERLA_ASSERT_GREATER_EQUAL(...) ((void)0)
#define WALBERLA_ASSERT_NOT_IDENTICAL(...) ((void)0)
#define WALBERLA_ABORT(msg) __builtin_trap()
