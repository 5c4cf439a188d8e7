// Many problems at once (hgg_batch_*) and the serving loop over a batch
// (hgg_server_*).
#include <algorithm>
#include <cmath>
#include <cstring>
#include <memory>
#include <mutex>
#include <string>
#include <vector>

#include "handle.cuh"

using namespace hgg;

// grouped execution of many problems (hgg_batch_*)
#include "batch_exec.cuh"
// serving loop over a batch (hgg_server_*)
#include "server.cuh"
