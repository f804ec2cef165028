"""Test infrastructure: CPU restatements of the reference path (the oracle).

Only tests, the smoke check and the benchmark's CPU-baseline arm import this
package; the product package never does.
"""
