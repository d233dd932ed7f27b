"""Oracle: CPU restatement of the reference's spectral path -- TEST INFRASTRUCTURE ONLY.

Nothing in the product package (mlx_signal_b200) imports this package. Only tests/, the
smoke() check in __graft_entry__.py and bench.py's CPU legs (cpu_baseline and
`--impl reference`) may use it, and only as the checker / CPU baseline.

Contents
--------
* ``cpu_reference``: the reference's own CPU route for the spectral functions. mlx-signal sends
  work to ``scipy.signal`` on its CPU path (src/mlx_signal_processing/spectral.py:433-450,
  654-669, 714-731, 842-858; routing rule _config.py:94-100); the reference's tests use the same
  calls in float64 as their golden oracle (tests/test_spectral.py:1-8). Adds a process-pool
  driver that splits channels over host cores (channels are independent, so this is exact).
* ``restate``: a NumPy restatement of the reference's kernel algorithms -- the packed-real
  Stockham FFT with its untangle (src/mlx_signal_processing/_stft_metal.py:33-147), the grouped
  segment accumulation (:426-557, :620-746), the inverse repack + gather overlap-add
  (:753-887), the three-pass large FFT index maps (_fourstep_metal.py:15-26, 90-185, 206-215)
  and the large-n real untangle (_fourstep.py:195-231, 360-408).

Parity pinning: the reference ships no stored vectors -- its tests compare against float64
scipy/numpy computed in-test. ``restate`` is checked against float64 scipy on the reference's
own test cases (tests/test_oracle.py), and the golden fixtures under tests/golden/ are float64
scipy outputs of seeded inputs produced by tests/golden/make_golden.py.
"""
