#pragma once
// Test-infrastructure shim, project-written.  The reference's inc/util.hpp
// includes <papi.h>, but nothing on the octree search path uses a PAPI symbol.
