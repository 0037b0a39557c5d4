/* hmm_port.c -- ORACLE: restatement of the integer HMM profile DP (filled in with that path). */
