// Continuous-batching request loop; filled in below the engine.
#include "server.h"
