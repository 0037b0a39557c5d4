/* gapless_port.c -- ORACLE: restatement of the gapless prefilter (filled in with that path). */
