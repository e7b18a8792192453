// flash_plain_nc12.cu -- the plain FP64 FIM flash kernels for 12 hydrocarbon
// components (flash_plain_inst.cuh).
#define OCPF_NC 12
#include "flash_plain_inst.cuh"
