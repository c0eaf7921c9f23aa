// Continuous-batching request loop (see server.cu).
#pragma once
