// flash_phased_nc9.cu -- the batched FIM flash kernels for 9 hydrocarbon
// components and their launch sequence (flash_phased_inst.cuh).
#define OCPF_NC 9
#include "flash_phased_inst.cuh"
