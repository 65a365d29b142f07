// Step<float>: the mixed form of the step and every kernel it launches, instantiated here
// so that the two precision forms compile in parallel.
#include "spo_host.cuh"

namespace spo_host {

template class Step<float>;

std::unique_ptr<StepBase> make_step_f32(const spo_desc& d, const Sizes& s, cudaStream_t stream) {
  return std::make_unique<Step<float>>(d, s, stream);
}

}  // namespace spo_host
