#pragma once
#include "vtk_stub.h"
