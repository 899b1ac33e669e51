// Compiles the reference's src/cpu/spline.cpp where it lies (see ref_dispatch.h).
#include "ref_dispatch.h"
#include "cpu/spline.cpp"
