// The oracle binds the FP32 regularisers only.
template class HuberRegularizer_CPU<float>;
