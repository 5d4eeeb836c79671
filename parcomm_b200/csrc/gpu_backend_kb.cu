// The CUDA backend compiled for KoalaBear^4 with signed 16-bit payloads.
#define QF_FIELD_KB 1
#include "gpu_backend.cu"
