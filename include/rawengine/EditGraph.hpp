// Same include name as the reference header EditGraph.hpp; the render-path
// subset (operation records, the operation factory, TileCache) lives in EditOps.hpp.
#pragma once
#include "EditOps.hpp"
