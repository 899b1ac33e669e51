// Compiles the reference's src/cpu/dcf.cpp where it lies (see ref_dispatch.h).
#include "ref_dispatch.h"
#include "cpu/dcf.cpp"
