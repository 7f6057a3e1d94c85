/* Host-only link stub for building the reference's src/common/mr_config.cpp
 * on its own (TEST INFRASTRUCTURE ONLY): that file calls the backend hook
 * mr_backend_clear_error (src/cuda/mr_backend_cuda.cu:21 of the reference, a
 * C++ function), which only resets CUDA's last error and has nothing to do on
 * a host-only build. */
void mr_backend_clear_error(void) {}
