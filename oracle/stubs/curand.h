/* Host-only stand-in for <curand.h> (oracle recipe only); nothing from it is used. */
