// ref_cuda_stub.cpp -- TEST INFRASTRUCTURE ONLY. The reference's host timing instrument
// (interFoam/inter_phase_time.cuh) calls cudaDeviceSynchronize, but only when BRAE_INTER_PHASE_TIME
// is set, which nothing here does. This no-op stands in so the reference's host-only solver code
// links without the CUDA runtime; it is bound inside libref.so only (-Bsymbolic, loaded RTLD_LOCAL).
extern "C" int cudaDeviceSynchronize(void) { return 0; }
