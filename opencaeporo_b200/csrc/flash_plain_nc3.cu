// flash_plain_nc3.cu -- the plain FP64 FIM flash kernels for 3 hydrocarbon
// components (flash_plain_inst.cuh).
#define OCPF_NC 3
#include "flash_plain_inst.cuh"
