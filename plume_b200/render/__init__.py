"""The volume render: the B200 implementation behind chadmv/plume's `plume.render` entry points."""
