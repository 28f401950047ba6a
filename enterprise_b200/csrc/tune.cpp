// Autotuner (placeholder).
#include "ent_internal.h"
