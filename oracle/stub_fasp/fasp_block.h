/* TEST INFRASTRUCTURE ONLY: see fasp.h. */
