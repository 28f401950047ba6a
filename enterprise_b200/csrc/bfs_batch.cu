// Bitwise multi-source BFS (placeholder until the batched kernels land).
#include "dev_graph.h"
namespace ent {
struct BatchWorkspace {};
void destroy_batch_workspace(BatchWorkspace* w) { delete w; }
}  // namespace ent
using namespace ent;
extern "C" {
int ent_bfs_batch(ent_graph*, const int32_t*, int32_t, int32_t*, ent_stats*) {
  return fail(ENT_ERR_UNSUPPORTED, "batched traversal not built yet");
}
int ent_bfs_batch_device(ent_graph*, const int32_t*, int32_t, int32_t*, void*, ent_stats*) {
  return fail(ENT_ERR_UNSUPPORTED, "batched traversal not built yet");
}
int ent_bfs_multi(ent_graph* const*, int32_t, const int32_t*, const int32_t*, int32_t* const*) {
  return fail(ENT_ERR_UNSUPPORTED, "multi-graph traversal not built yet");
}
}
