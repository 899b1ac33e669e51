/* Aliases kept from include/FastFss/cuda/onehot.h:13-18 of the reference. */
#ifndef FAST_FSS_CUDA_ONEHOT_H
#define FAST_FSS_CUDA_ONEHOT_H

#include "ottt.h"

#define FastFss_cuda_onehotKeyGen  FastFss_cuda_otttKeyGen
#define FastFss_cuda_onehotLutEval FastFss_cuda_otttLutEval

#endif
