"""The live viewer's device compute (mirrors chadmv/plume src/plume/view): the look, the centre ray's depth,
the slice plane, the boundary layers and the frame cache's float16 casts. The window (imgui + OpenGL) is not
part of this package: these produce the display bytes it would show."""
