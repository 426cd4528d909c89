// Forced include for pe built with the B200 collision system and pe's DEM response: pe's own
// sources and World, with the step run by libpe_b200 (the drop-in's test build).
#include "config_common.h"
#define pe_CONSTRAINT_SOLVER pe::response::DEMSolver
#include <pe_b200_pe/pe_b200_pe_config.h>
