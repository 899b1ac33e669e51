// Compiles the reference's src/dcf.cpp (host-side key/cache size functions) where it lies.
#include "ref_dispatch.h"
#include "dcf.cpp"
