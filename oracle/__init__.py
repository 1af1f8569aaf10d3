"""CPU oracle of the DTB hot path -- test infrastructure only (see lif_oracle.py)."""
