// The primary fields of one grid cell as the reference's field struct holds
// them (fields.hh:1-36). On the B200 path the fields live on the device;
// fluid_2d::sync_fields() fills a host copy of u, v and p in this layout for
// the output and restart routines and for callers that read fbase/fm.
#ifndef VDI_HOST_FIELDS_HH
#define VDI_HOST_FIELDS_HH

struct field {
    double u;
    double v;
    double p;
    inline void clear_main() { u = v = p = 0; }
    /** Packs u, v, p into an array (the restart-file record). */
    inline void pack(double*& pp) {
        *(pp++) = u;
        *(pp++) = v;
        *(pp++) = p;
    }
    inline void unpack(double*& pp) {
        u = *(pp++);
        v = *(pp++);
        p = *(pp++);
    }
};

#endif
