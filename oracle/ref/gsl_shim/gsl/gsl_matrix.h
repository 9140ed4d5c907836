/* Stand-in: included by the reference solver, no symbol used. */
