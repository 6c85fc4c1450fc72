"""Case generators: the reference's cases (close-packed 3-D lattice) and the
benchmark variants (true 2-D square and 3-D cubic lattices)."""
