// Compiles the reference's src/cpu/prng.cpp where it lies (see ref_dispatch.h).
#include "ref_dispatch.h"
#include "cpu/prng.cpp"
