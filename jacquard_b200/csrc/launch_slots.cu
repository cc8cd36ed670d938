// Launch slots: which grid-barrier / status slot a launch uses.
//
// Each interpreter keeps its grid-barrier counters and its error status in
// module memory, BAR_SLOTS entries per device.  A launch takes the slot of
// the stream it is issued on: launches on one stream run one after another
// and share it, launches on different streams of one device get different
// slots, so their barriers and statuses never mix.  The table is per process
// and never shrinks; a stream handle keeps its slot for the life of the
// process (a destroyed stream's handle that the runtime hands out again maps
// to the same slot, which is safe once the old stream's work has finished).
// The legacy default stream (NULL or cudaStreamLegacy) is one key.
// cudaStreamPerThread is one handle for every host thread, so launches on it
// from several threads share a slot and must not overlap.
#include <mutex>

#include "sim_common.cuh"

namespace jqk {

namespace {
struct SlotKey {
  int device;
  void *stream;
  bool used;
};
SlotKey g_keys[BAR_SLOTS];
std::mutex g_keys_mu;
}  // namespace

int launch_slot(void *stream, bool assign) {
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess) return -1;
  if (stream == (void *)cudaStreamLegacy) stream = nullptr;
  std::lock_guard<std::mutex> lk(g_keys_mu);
  int free_i = -1;
  for (int i = 0; i < BAR_SLOTS; ++i) {
    if (g_keys[i].used) {
      if (g_keys[i].device == dev && g_keys[i].stream == stream) return i;
    } else if (free_i < 0) {
      free_i = i;
    }
  }
  if (!assign || free_i < 0) return -1;
  g_keys[free_i] = SlotKey{dev, stream, true};
  return free_i;
}

}  // namespace jqk
