FOREACH_CONFIG(reference_config)
FOREACH_CONFIG(haswell_config)
FOREACH_CONFIG(zen_config)

#undef FOREACH_CONFIG
