// Step<double>: the FP64 form of the step and every kernel it launches, instantiated here
// so that the two precision forms compile in parallel.
#include "spo_host.cuh"

namespace spo_host {

template class Step<double>;

std::unique_ptr<StepBase> make_step_f64(const spo_desc& d, const Sizes& s, cudaStream_t stream) {
  return std::make_unique<Step<double>>(d, s, stream);
}

}  // namespace spo_host
