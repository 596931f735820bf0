"""bem_b200 -- B200-native backend for the specific_particle_tracer hot path."""
