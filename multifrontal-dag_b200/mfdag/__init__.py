"""B200 numeric phase for the supernodal multifrontal Cholesky solver."""
