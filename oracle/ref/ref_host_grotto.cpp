// Compiles the reference's src/grotto.cpp (host-side key/cache size functions) where it lies.
#include "ref_dispatch.h"
#include "grotto.cpp"
