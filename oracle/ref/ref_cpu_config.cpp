// Compiles the reference's src/cpu/config.cpp where it lies (see ref_dispatch.h).
#include "ref_dispatch.h"
#include "cpu/config.cpp"
