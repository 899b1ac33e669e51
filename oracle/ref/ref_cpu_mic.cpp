// Compiles the reference's src/cpu/mic.cpp where it lies (see ref_dispatch.h).
#include "ref_dispatch.h"
#include "cpu/mic.cpp"
