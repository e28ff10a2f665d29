// Stand-in for GDAL's ogrsf_frmts.h so the unmodified reference sources
// compile into the oracle binary without GDAL. TEST INFRASTRUCTURE ONLY.
// The only symbol the step-loop sources need from it is GDALAllRegister();
// shapefile release polygons (which need OGR) are not supported by the oracle.
//
// The real header (through cpl_port.h) includes <stdlib.h> and <math.h>. In a
// C++ translation unit those bring the floating-point overloads of abs() into
// the global namespace, and simulation.cpp:403 relies on that: it calls an
// unqualified abs() on a double. Without these two includes that call would
// bind to C's int abs() and truncate.
#pragma once
#include <math.h>
#include <stdlib.h>
inline void GDALAllRegister() {}
