// Test-infrastructure shim: inert stand-ins for the VTK classes that the
// reference's Model::saveVTK names, so Model.cpp compiles without VTK.  The
// oracle never calls saveVTK; every method here does nothing.
#pragma once
#include "vtk_inert.h"
