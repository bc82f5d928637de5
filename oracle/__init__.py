"""CPU oracle of the Vidyut3d step -- test infrastructure only (see oracle.py)."""
