// Engine interface of the serving loop (zfpb_serve.cpp).
#pragma once

#include "zfpb_engine.h"

namespace zfpb {

struct Server;

// A finished request.
struct ServeDone {
  u64 tag;
  u64 result;         // stream bytes written / consumed, 0 on failure
  int status;         // Status of the request
  double queue_ms;    // submit -> launch
  double latency_ms;  // submit -> result available on the host
};

// budget: device bytes that admitted requests may hold at once (their fields,
// streams and batch scratch); lanes: batches in flight at once (0: 4);
// max_batch: requests per batch (0: 4096); batch_bytes: uncompressed bytes
// per batch, a larger request running alone (0: 64 MiB).
Server* server_create(u64 budget, int lanes, size_t max_batch, u64 batch_bytes);
// false when the request alone exceeds the budget.
bool server_submit(Server* s, const BatchJob& job, bool decompress, u64 tag);
// Finished requests (up to max), waiting up to wait_ms for the first.
size_t server_poll(Server* s, ServeDone* out, size_t max, int wait_ms);
// Submitted requests not yet returned by server_poll.
size_t server_outstanding(Server* s);
// Finishes the submitted work, then frees the server.
void server_destroy(Server* s);

}  // namespace zfpb
