// flash_plain_nc9.cu -- the plain FP64 FIM flash kernels for 9 hydrocarbon
// components (flash_plain_inst.cuh).
#define OCPF_NC 9
#include "flash_plain_inst.cuh"
