/* Stand-in: included by the reference's sources.c; no symbol used. */
