// flash_plain_nc6.cu -- the plain FP64 FIM flash kernels for 6 hydrocarbon
// components (flash_plain_inst.cuh).
#define OCPF_NC 6
#include "flash_plain_inst.cuh"
