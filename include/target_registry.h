/*
 * target_registry.h -- target contexts known to the config layer.
 *
 * Mirrors the reference's targets/target_registry.h:6-12: each target is
 * declared as `extern const mublis_context_t <name>;`.  The B200 build links
 * exactly one target, b200_context (CPU targets of the reference are not part
 * of this library).
 */
#ifndef MUBLIS_TARGET_REGISTRY_H
#define MUBLIS_TARGET_REGISTRY_H

#include "mublis_instantiate.h"

#define REGISTER_TARGET_CONTEXT(name) extern const mublis_context_t name;

#ifdef __cplusplus
extern "C" {
#endif

REGISTER_TARGET_CONTEXT(b200_context)

#ifdef __cplusplus
}
#endif

#endif
