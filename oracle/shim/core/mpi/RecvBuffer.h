// Project-written stand-in for waLBerla's MPI receive buffer (see SendBuffer.h).
#pragma once
namespace walberla { namespace mpi {
template <typename T = unsigned char> struct GenericRecvBuffer {
  template <typename V> GenericRecvBuffer& operator>>(V&) { return *this; }
};
typedef GenericRecvBuffer<> RecvBuffer;
}}  // namespace walberla::mpi
