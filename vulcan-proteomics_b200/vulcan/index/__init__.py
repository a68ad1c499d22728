"""L1 proteome index: digestion, paired decoys, hash-assigned peptidoform ids, mass-sorted rows."""
