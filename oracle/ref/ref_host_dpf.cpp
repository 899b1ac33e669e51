// Compiles the reference's src/dpf.cpp (host-side key/cache size functions) where it lies.
#include "ref_dispatch.h"
#include "dpf.cpp"
