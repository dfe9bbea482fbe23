"""B200-native finite-element assembly for EMerge: drop-ins for its hot
paths, all computing on the GPU through ``libemgpu.so`` (``include/emgpu.h``).

Modules (imported on use, so ``import emerge_b200`` stays light):

* ``assembly``     -- ``tet_mass_stiffness_matrices`` and ``GpuCSCMapping``
  (curlcurl.py / csc_cast.py: Nedelec-2 K, M and A = K - k0^2 M in CSC)
* ``robin``        -- ``RobinTerm``: port / Robin terms, the port forcing
  vector, the second-order ABC correction (robinbc.py, robin_abc_order2.py)
* ``sweep``        -- ``FrequencySweep``: K and M resident, A(f) per frequency
* ``serving``      -- ``AssemblyServer``: batched assembly jobs under an HBM budget
* ``partition``    -- column shards of A, one per GPU
* ``solve_dofs``   -- ``SolveSubmatrix``: the solve-DoF system on the device
  and its solve
* ``postprocess``  -- field at points and S-parameter port integrals
* ``heat``         -- Lagrange-2 heat conduction and ``GpuCOOMapping``
"""
__version__ = "0.1.0"
