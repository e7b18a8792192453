// flash_phased_nc3.cu -- the batched FIM flash kernels for 3 hydrocarbon
// components and their launch sequence (flash_phased_inst.cuh).
#define OCPF_NC 3
#include "flash_phased_inst.cuh"
