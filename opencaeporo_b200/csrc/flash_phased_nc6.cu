// flash_phased_nc6.cu -- the batched FIM flash kernels for 6 hydrocarbon
// components and their launch sequence (flash_phased_inst.cuh).
#define OCPF_NC 6
#include "flash_phased_inst.cuh"
