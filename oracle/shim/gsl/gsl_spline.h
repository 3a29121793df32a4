/* ORACLE ONLY: GSL stand-in; amber includes this header but calls nothing from it. */
