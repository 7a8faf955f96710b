/* Included by the reference but unused (its MapVector is robin_map). */
