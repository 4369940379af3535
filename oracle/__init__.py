"""FP64 CPU oracle of align_group_to_template: test infrastructure, never product code."""
