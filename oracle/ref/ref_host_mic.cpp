// Compiles the reference's src/mic.cpp (host-side key/cache size functions) where it lies.
#include "ref_dispatch.h"
#include "mic.cpp"
