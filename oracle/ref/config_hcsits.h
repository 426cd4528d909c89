// Forced include for the hard-contact (HCSITS) build of the compiled reference (oracle only).
#include "config_common.h"
#define pe_CONSTRAINT_SOLVER pe::response::HardContactSemiImplicitTimesteppingSolvers
