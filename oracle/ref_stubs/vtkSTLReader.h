#include "stub_vtk.h"
