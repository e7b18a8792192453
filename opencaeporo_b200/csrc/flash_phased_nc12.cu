// flash_phased_nc12.cu -- the batched FIM flash kernels for 12 hydrocarbon
// components and their launch sequence (flash_phased_inst.cuh).
#define OCPF_NC 12
#include "flash_phased_inst.cuh"
