/* SU trace type for the oracle build. TEST INFRASTRUCTURE ONLY.
 *
 * The 240-byte header follows the public SEG-Y rev.0 trace-header byte
 * positions (bytes 1-180) plus the documented SU extension fields d1, f1, d2,
 * f2, ungpow, unscale, ntr, mark (bytes 181-212). The layout is a file format
 * and must match byte for byte; the field names are the SU names the
 * reference's sources use. */
#ifndef ORACLE_SUSHIM_SEGY_H
#define ORACLE_SUSHIM_SEGY_H

#define SU_NFLTS 32767
#define HDRBYTES 240

typedef struct {
  int tracl;               /*   0 */
  int tracr;               /*   4 */
  int fldr;                /*   8 */
  int tracf;               /*  12 */
  int ep;                  /*  16 */
  int cdp;                 /*  20 */
  int cdpt;                /*  24 */
  short trid;              /*  28 */
  short nvs;               /*  30 */
  short nhs;               /*  32 */
  short duse;              /*  34 */
  int offset;              /*  36 */
  int gelev;               /*  40 */
  int selev;               /*  44 */
  int sdepth;              /*  48 */
  int gdel;                /*  52 */
  int sdel;                /*  56 */
  int swdep;               /*  60 */
  int gwdep;               /*  64 */
  short scalel;            /*  68 */
  short scalco;            /*  70 */
  int sx;                  /*  72 */
  int sy;                  /*  76 */
  int gx;                  /*  80 */
  int gy;                  /*  84 */
  short counit;            /*  88 */
  short wevel;             /*  90 */
  short swevel;            /*  92 */
  short sut;               /*  94 */
  short gut;               /*  96 */
  short sstat;             /*  98 */
  short gstat;             /* 100 */
  short tstat;             /* 102 */
  short laga;              /* 104 */
  short lagb;              /* 106 */
  short delrt;             /* 108 */
  short muts;              /* 110 */
  short mute;              /* 112 */
  unsigned short ns;       /* 114 */
  unsigned short dt;       /* 116 */
  short gain;              /* 118 */
  short igc;               /* 120 */
  short igi;               /* 122 */
  short corr;              /* 124 */
  short sfs;               /* 126 */
  short sfe;               /* 128 */
  short slen;              /* 130 */
  short styp;              /* 132 */
  short stas;              /* 134 */
  short stae;              /* 136 */
  short tatyp;             /* 138 */
  short afilf;             /* 140 */
  short afils;             /* 142 */
  short nofilf;            /* 144 */
  short nofils;            /* 146 */
  short lcf;               /* 148 */
  short hcf;               /* 150 */
  short lcs;               /* 152 */
  short hcs;               /* 154 */
  short year;              /* 156 */
  short day;               /* 158 */
  short hour;              /* 160 */
  short minute;            /* 162 */
  short sec;               /* 164 */
  short timbas;            /* 166 */
  short trwf;              /* 168 */
  short grnors;            /* 170 */
  short grnofr;            /* 172 */
  short grnlof;            /* 174 */
  short gaps;              /* 176 */
  short otrav;             /* 178 */
  float d1;                /* 180 */
  float f1;                /* 184 */
  float d2;                /* 188 */
  float f2;                /* 192 */
  float ungpow;            /* 196 */
  float unscale;           /* 200 */
  int ntr;                 /* 204 */
  short mark;              /* 208 */
  short shortpad;          /* 210 */
  short unass[14];         /* 212 .. 239 */
  float data[SU_NFLTS];    /* 240 */
} segy;

#endif
