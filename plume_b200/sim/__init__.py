"""The fluid step: the B200 implementation behind chadmv/plume's `plume.sim` entry points."""
