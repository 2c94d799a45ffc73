// Forwarding header: see _tbb_stub.h (oracle build only).
#include "_tbb_stub.h"
