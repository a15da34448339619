"""seisfem_b200: B200-native mass-lumped explicit time stepping for SeisFEM."""
