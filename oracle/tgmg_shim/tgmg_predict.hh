/* V-cycle bookkeeping for the clean-room TGMG-API shim (test infrastructure,
 * see tgmg_config.hh). The reference reads two things from it:
 * vcount_extra() for the machine-readable per-frame line (fluid_2d.cc:286-287)
 * and avg_iters(true) for the average per solve, which also resets the
 * counters (mgs_common.hh:62-65, fluid_2d.cc:288-290). */
#ifndef TGMG_PREDICT_HH
#define TGMG_PREDICT_HH

struct tgmg_predict {
    /** V-cycles performed since the last reset. */
    long vcount;
    /** Solves performed since the last reset. */
    long scount;
    /** V-cycles of the most recent solve. */
    int last;
    tgmg_predict() : vcount(0), scount(0), last(0) {}
    inline void record(int k) {vcount+=k;scount++;last=k;}
    /** Total V-cycles since the last reset. */
    inline int vcount_extra() {return static_cast<int>(vcount);}
    /** Average V-cycles per solve since the last reset.
     * \param[in] reset whether to clear the counters afterwards. */
    inline float avg_iters(bool reset) {
        float a=scount>0?static_cast<float>(vcount)/scount:0.f;
        if(reset) vcount=scount=0;
        return a;
    }
};

#endif
