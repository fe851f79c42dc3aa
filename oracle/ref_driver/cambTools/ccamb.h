/* ccamb.h — empty stand-in for the reference's CAMB bindings, which the
 * serial() driver only calls when built without NOPYTHON.  TEST
 * INFRASTRUCTURE ONLY. */
