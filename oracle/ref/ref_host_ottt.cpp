// Compiles the reference's src/ottt.cpp (host-side key/cache size functions) where it lies.
#include "ref_dispatch.h"
#include "ottt.cpp"
