// Stand-in for the reference's GPUHandler.h in the build of its GPU engine
// (GPUEngine.cu includes it but uses nothing from it; the real header needs
// hybridsys, TBB and the FPGA layer).  TEST INFRASTRUCTURE.
#pragma once
#include "Datatypes.h"
