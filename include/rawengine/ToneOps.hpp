// Same include name as the reference header ToneOps.hpp; the declarations of the
// render-path subset live in Operators.hpp.
#pragma once
#include "Operators.hpp"
