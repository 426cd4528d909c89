// Forced include for the DEM build of the compiled reference (oracle only).
#include "config_common.h"
#define pe_CONSTRAINT_SOLVER pe::response::DEMSolver
