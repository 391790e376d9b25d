// Stand-in header for the absent OpenWQ submodule (oracle build only).
#include "OpenWQ_global.h"
