/* empty stub: the reference includes readline but never calls it (util/Util.h:69-70) */
