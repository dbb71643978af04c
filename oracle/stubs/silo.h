/* No-op stand-in for the Silo I/O library, used only when building the
 * reference code as a test oracle.  The reference writes VisIt/Silo files from
 * GridNode::output (grid/grid_node.cpp:1422-1487); the oracle never calls that
 * path, so every entry point here only has to exist and return quietly. */
#ifndef ORACLE_SILO_STUB_H
#define ORACLE_SILO_STUB_H

typedef struct DBfile_s { int unused; } DBfile;
typedef struct DBoptlist_s { int unused; } DBoptlist;

#define DB_CLOBBER 0
#define DB_LOCAL 0
#define DB_PDB 0
#define DB_HDF5 0
#define DB_READ 0
#define DB_UNKNOWN 0
#define DB_ZONETYPE_HEX 12
#define DB_DOUBLE 20
#define DB_FLOAT 19
#define DB_INT 16
#define DB_ZONECENT 111
#define DB_NODECENT 110
#define DBOPT_TIME 267
#define DBOPT_DTIME 268
#define DBOPT_CYCLE 266

static inline DBoptlist* DBMakeOptlist(int) { static DBoptlist o; return &o; }
static inline int DBAddOption(DBoptlist*, int, void*) { return 0; }
static inline int DBFreeOptlist(DBoptlist*) { return 0; }
static inline DBfile* DBCreate(const char*, int, int, const char*, int) { static DBfile f; return &f; }
static inline DBfile* DBOpen(const char*, int, int) { return 0; }
static inline int DBPutZonelist2(DBfile*, const char*, int, int, const int*, int, int, int, int,
                                 const int*, const int*, const int*, int, DBoptlist*) { return 0; }
static inline int DBPutUcdmesh(DBfile*, const char*, int, char**, float**, int, int, const char*,
                               const char*, int, DBoptlist*) { return 0; }
static inline int DBPutUcdmesh(DBfile*, const char*, int, char**, double**, int, int, const char*,
                               const char*, int, DBoptlist*) { return 0; }
static inline int DBPutUcdvar1(DBfile*, const char*, const char*, float*, int, void*, int, int, int,
                               DBoptlist*) { return 0; }
static inline int DBPutUcdvar1(DBfile*, const char*, const char*, double*, int, void*, int, int, int,
                               DBoptlist*) { return 0; }
static inline int DBClose(DBfile*) { return 0; }

/* Read side, only named by Binary::input (binary/binary.cpp:1098-1169),
 * which the oracle never calls. */
typedef struct DBzonelist_s { int* nodelist; int nzones; int lnodelist; } DBzonelist;
typedef struct DBucdmesh_s {
    void* min_extents;
    void* max_extents;
    void* coords[3];
    DBzonelist* zones;
    int nnodes;
    double time;
} DBucdmesh;
typedef struct DBucdvar_s { void** vals; } DBucdvar;
static inline DBucdmesh* DBGetUcdmesh(DBfile*, const char*) { return 0; }
static inline DBucdvar* DBGetUcdvar(DBfile*, const char*) { return 0; }
static inline void DBFreeUcdmesh(DBucdmesh*) {}
static inline void DBFreeUcdvar(DBucdvar*) {}

#endif
