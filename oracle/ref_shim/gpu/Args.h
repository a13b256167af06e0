// Stand-in for the reference's Args.h in the build of its GPU engine
// (GPUEngine.cu includes it but uses nothing from it; the real header needs
// boost::program_options).  TEST INFRASTRUCTURE.
#pragma once
#include "Datatypes.h"
