// Include-path stand-in for the numerics library header structures/graph/graph.hpp that
// MarkovKit's programs include: num::graph (an explicit weighted voxel graph) is declared by the
// facade, so a program written against the reference builds with -I include/mk.
#pragma once

#include "../../markovkit.hpp"
