"""B200-native SolTrace coretrace: CUDA trace behind the stapi.h C ABI."""
