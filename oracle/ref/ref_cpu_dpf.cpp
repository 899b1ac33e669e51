// Compiles the reference's src/cpu/dpf.cpp where it lies (see ref_dispatch.h).
#include "ref_dispatch.h"
#include "cpu/dpf.cpp"
