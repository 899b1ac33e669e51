// Compiles the reference's src/cpu/ottt.cpp where it lies (see ref_dispatch.h).
#include "ref_dispatch.h"
#include "cpu/ottt.cpp"
