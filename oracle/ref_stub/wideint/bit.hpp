// See wideint.hpp in this directory.
#pragma once
#include "wideint.hpp"
