// Policy selectors of the GAS Program contract. The names and values are the
// reference's (GASengine/Enums.h:2-25) so that Program structs written against
// the reference compile unchanged against this engine.
#pragma once

enum SrcVertex { SINGLE, ALL };

enum GatherEdges { NO_GATHER_EDGES, GATHER_IN_EDGES, GATHER_OUT_EDGES, GATHER_ALL_EDGES };

enum ExpandEdges { NO_EXPAND_EDGES, EXPAND_IN_EDGES, EXPAND_OUT_EDGES, EXPAND_ALL_EDGES };

enum ApplyVertices { NO_APPLY_VERTICES, APPLY_ALL, APPLY_FRONTIER };

enum PostApplyVertices { NO_POST_APPLY_VERTICES, POST_APPLY_ALL, POST_APPLY_FRONTIER };
