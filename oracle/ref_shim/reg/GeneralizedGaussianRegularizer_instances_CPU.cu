// The oracle binds the FP32 regularisers only.
template class GeneralizedGaussianRegularizer_CPU<float>;
