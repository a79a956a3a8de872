"""Sheet assembly and the numbers file on the device (mirrors chadmv/plume src/plume/sheet and
src/plume/report/numbers.py)."""
