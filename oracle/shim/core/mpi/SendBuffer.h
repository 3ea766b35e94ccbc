// Project-written stand-in for waLBerla's MPI send buffer: an empty stream type, so that
// the (unused) serialisation helpers of the reference's PointND header compile.
#pragma once
namespace walberla { namespace mpi {
struct OptimalGrowth {};
template <typename T = unsigned char, typename G = OptimalGrowth> struct GenericSendBuffer {
  template <typename V> GenericSendBuffer& operator<<(const V&) { return *this; }
};
typedef GenericSendBuffer<> SendBuffer;
}}  // namespace walberla::mpi
