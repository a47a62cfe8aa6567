// Evaluation of a sequence of states held in HOST memory with the copies
// overlapped: functionals::total (include/dft/functionals/functionals.hpp:
// 64-95) once per state, the host->device copy of state i+1 and the
// device->host copy of the forces of state i-1 running on their own streams
// while state i is evaluated.
//
// Two device slots (rho, V_ext, force, scalars) alternate between the
// states.  Per state i in slot s = i % 2:
//   copy-in stream : wait until evaluation i-2 has read slot s, copy rho_i
//                    (and V_ext_i) in, record in_ready[s];
//   engine stream  : wait in_ready[s] and until the forces of state i-2 have
//                    left slot s, evaluate, record eval_done[s];
//   copy-out stream: wait eval_done[s], copy force_i and the scalars out,
//                    record out_done[s].
// The host waits once, after the last state.  With page-locked host
// buffers the three streams overlap (PCIe is full duplex); with pageable
// ones the copies are staged by the driver and the result is the same.
#pragma once

#include "engine.cuh"

namespace cdft {

class HostStream {
 public:
  explicit HostStream(Engine& e);
  ~HostStream();
  HostStream(const HostStream&) = delete;
  HostStream& operator=(const HostStream&) = delete;

  // count states.  rho[i], force[i]: B*S*N host doubles each (force[i] may
  // be NULL); vext: NULL (no field) or count pointers (entries may be NULL);
  // mu: count * B*S values; scalars: NULL or count * B*CDFT_SCALAR_COUNT.
  void run(int count, const double* const* rho, const double* const* vext, const double* mu, double* const* force,
           double* scalars);

 private:
  static constexpr int kSlots = 2;
  Engine& e_;
  size_t bytes_ = 0;  // one state: B*S*N doubles
  double* rho_[kSlots] = {};
  double* vext_[kSlots] = {};
  double* force_[kSlots] = {};
  double* scal_[kSlots] = {};
  cudaStream_t in_ = nullptr, out_ = nullptr;
  cudaEvent_t in_ready_[kSlots] = {}, eval_done_[kSlots] = {}, out_done_[kSlots] = {};
};

}  // namespace cdft
