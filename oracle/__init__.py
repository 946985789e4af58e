"""The oracle: a CPU restatement of zephyr's single-material step, used only
as the checker by the tests, the smoke check and the bench's CPU-baseline leg.
"""
