// Library identification.
#include "oceansar_b200.h"

extern "C" const char *ocs_version(void) { return "0.1.0"; }
