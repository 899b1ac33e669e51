// Compiles the reference's src/cpu/grotto.cpp where it lies (see ref_dispatch.h).
#include "ref_dispatch.h"
#include "cpu/grotto.cpp"
