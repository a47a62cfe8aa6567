#include "host_stream.cuh"

#include <cstring>
#include <stdexcept>

namespace cdft {

HostStream::HostStream(Engine& e) : e_(e) {
  bytes_ = sizeof(double) * (size_t)e.batch() * e.species() * e.points();
  for (int s = 0; s < kSlots; ++s) {
    CDFT_CUDA(cudaMalloc(&rho_[s], bytes_));
    CDFT_CUDA(cudaMalloc(&force_[s], bytes_));
    CDFT_CUDA(cudaMalloc(&scal_[s], sizeof(double) * e.batch() * kScalarCount));
    CDFT_CUDA(cudaEventCreateWithFlags(&in_ready_[s], cudaEventDisableTiming));
    CDFT_CUDA(cudaEventCreateWithFlags(&eval_done_[s], cudaEventDisableTiming));
    CDFT_CUDA(cudaEventCreateWithFlags(&out_done_[s], cudaEventDisableTiming));
  }
  CDFT_CUDA(cudaStreamCreateWithFlags(&in_, cudaStreamNonBlocking));
  CDFT_CUDA(cudaStreamCreateWithFlags(&out_, cudaStreamNonBlocking));
}

HostStream::~HostStream() {
  for (int s = 0; s < kSlots; ++s) {
    for (double* q : {rho_[s], vext_[s], force_[s], scal_[s]})
      if (q) cudaFree(q);
    for (cudaEvent_t ev : {in_ready_[s], eval_done_[s], out_done_[s]})
      if (ev) cudaEventDestroy(ev);
  }
  if (in_) cudaStreamDestroy(in_);
  if (out_) cudaStreamDestroy(out_);
}

void HostStream::run(int count, const double* const* rho, const double* const* vext, const double* mu,
                     double* const* force, double* scalars) {
  if (count < 0) throw std::invalid_argument("host stream: count must be non-negative");
  if (count == 0) return;
  if (!rho || !mu) throw std::invalid_argument("host stream: rho and mu are required");
  for (int i = 0; i < count; ++i)
    if (!rho[i]) throw std::invalid_argument("host stream: every rho pointer is required");
  bool any_v = false;
  if (vext)
    for (int i = 0; i < count; ++i) any_v = any_v || vext[i] != nullptr;
  if (any_v && !vext_[0])
    for (int s = 0; s < kSlots; ++s) CDFT_CUDA(cudaMalloc(&vext_[s], bytes_));
  const int B = e_.batch(), S = e_.species();
  const size_t sc_per = (size_t)B * kScalarCount;
  // page-locked staging of the scalars: a device->host copy into pageable
  // memory would hold the host until it completes and stall the pipeline
  double* sc_pin = nullptr;
  CDFT_CUDA(cudaHostAlloc(&sc_pin, sizeof(double) * sc_per * count, cudaHostAllocDefault));
  cudaStream_t ev_st = e_.stream();
  try {
    for (int i = 0; i < count; ++i) {
      const int s = i % kSlots;
      const bool v_here = vext && vext[i];
      if (i >= kSlots) CDFT_CUDA(cudaStreamWaitEvent(in_, eval_done_[s], 0));
      CDFT_CUDA(cudaMemcpyAsync(rho_[s], rho[i], bytes_, cudaMemcpyHostToDevice, in_));
      if (v_here) CDFT_CUDA(cudaMemcpyAsync(vext_[s], vext[i], bytes_, cudaMemcpyHostToDevice, in_));
      CDFT_CUDA(cudaEventRecord(in_ready_[s], in_));
      CDFT_CUDA(cudaStreamWaitEvent(ev_st, in_ready_[s], 0));
      if (i >= kSlots) CDFT_CUDA(cudaStreamWaitEvent(ev_st, out_done_[s], 0));
      e_.evaluate(rho_[s], v_here ? vext_[s] : nullptr, mu + (size_t)i * B * S, force_[s], scal_[s], ev_st);
      CDFT_CUDA(cudaEventRecord(eval_done_[s], ev_st));
      CDFT_CUDA(cudaStreamWaitEvent(out_, eval_done_[s], 0));
      if (force && force[i]) CDFT_CUDA(cudaMemcpyAsync(force[i], force_[s], bytes_, cudaMemcpyDeviceToHost, out_));
      CDFT_CUDA(cudaMemcpyAsync(sc_pin + sc_per * i, scal_[s], sizeof(double) * sc_per, cudaMemcpyDeviceToHost, out_));
      CDFT_CUDA(cudaEventRecord(out_done_[s], out_));
    }
    CDFT_CUDA(cudaStreamSynchronize(out_));
    CDFT_CUDA(cudaStreamSynchronize(ev_st));
    CDFT_CUDA(cudaStreamSynchronize(in_));
  } catch (...) {
    cudaStreamSynchronize(out_);
    cudaStreamSynchronize(ev_st);
    cudaStreamSynchronize(in_);
    cudaFreeHost(sc_pin);
    throw;
  }
  const bool failed = e_.take_error(ev_st);
  if (scalars && !failed) std::memcpy(scalars, sc_pin, sizeof(double) * sc_per * count);
  cudaFreeHost(sc_pin);
  if (failed) throw Error(-2 /* CDFT_ERR_RUNTIME */, "evaluation aborted: a bounded device wait timed out");
}

}  // namespace cdft
