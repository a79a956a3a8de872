"""Host-side recipe settings: the subset of chadmv/plume's recipe schema the fluid step and the volume render
read, with the same table and key names and defaults, so a reference recipe file drives this package as is."""
