// Compiles the reference's src/spline.cpp (host-side key/cache size functions) where it lies.
#include "ref_dispatch.h"
#include "spline.cpp"
